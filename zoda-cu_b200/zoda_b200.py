"""Python host binding of libzoda_b200.so (the C ABI in include/zoda_b200.h).

This is the host-side mirror of the reference's encode API for this path:
  * ``ntt_cuda`` / ``intt_cuda`` keep the argument meaning and the error
    behaviour of src/ntt/cuda.rs:99-131 (power-of-two n, stride >= n, whole
    polynomials; a CUDA failure raises with the error code);
  * ``PinnedSquare`` mirrors src/ntt/cuda.rs:34-97 (column-major pinned u32);
  * ``Context.extend`` is the fused device-resident extension that replaces
    ``encode_gpu`` (src/benchmarks/utils.rs:100-146) and ``extend``
    (src/zoda/babybear.rs:34-46) for k = n = side.

The library must be built (``make -C zoda-cu_b200``); there is no fallback:
every call here runs the CUDA kernels or raises.
"""
from __future__ import annotations

import ctypes
import json
import os

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "libzoda_b200.so")

P = 2013265921
ZODA_OK = 0
STATUS = {
    0: "ok", 1: "invalid argument", 2: "CUDA error", 3: "out of memory", 4: "unsupported shape",
    5: "over the admission budget", 6: "timed out", 7: "cancelled", 8: "invalid state",
}

# every symbol include/zoda_b200.h declares
EXPORTS = [
    "cuda_ntt", "cuda_intt", "cuda_host_alloc", "cuda_host_free",
    "zoda_status_string", "zoda_last_error", "zoda_ctx_create", "zoda_ctx_destroy", "zoda_max_side",
    "zoda_extend_device", "zoda_extend_host", "zoda_ctx_set_impl", "zoda_ctx_check", "zoda_selftest_bounded_wait",
    "zoda_ntt_device_noalloc", "zoda_batch_create", "zoda_batch_run", "zoda_batch_elements",
    "zoda_batch_destroy", "zoda_server_create", "zoda_server_submit", "zoda_server_wait",
    "zoda_server_release", "zoda_server_cancel", "zoda_server_get_stats", "zoda_server_destroy",
    "zoda_encode_device", "zoda_recover_device", "zoda_autotune", "zoda_plan_get", "zoda_plan_set",
    "zoda_plan_clear", "zoda_data_root_host", "zoda_rlc_coefficients_device", "zoda_rlc_rows_device",
    "zoda_rlc_check_device", "zoda_ctx_inject_fault",
]

_lib = None


class ZodaError(RuntimeError):
    def __init__(self, status: int, where: str, detail: str = ""):
        self.status = status
        super().__init__(f"{where}: {STATUS.get(status, status)}" + (f" ({detail})" if detail else ""))


class ZodaSquare(ctypes.Structure):
    _fields_ = [("d_in", ctypes.c_void_p), ("d_out", ctypes.c_void_p), ("k", ctypes.c_uint32),
                ("reserved", ctypes.c_uint32), ("cols", ctypes.c_uint64)]


class ZodaServerConfig(ctypes.Structure):
    _fields_ = [("hbm_budget_bytes", ctypes.c_uint64), ("max_inflight", ctypes.c_uint32),
                ("max_batch", ctypes.c_uint32)]


class ZodaRequestInfo(ctypes.Structure):
    _fields_ = [("d_out", ctypes.c_void_p), ("queue_ms", ctypes.c_double), ("latency_ms", ctypes.c_double),
                ("status", ctypes.c_int32), ("reserved", ctypes.c_int32)]


class ZodaServerStats(ctypes.Structure):
    _fields_ = [("submitted", ctypes.c_uint64), ("completed", ctypes.c_uint64), ("cancelled", ctypes.c_uint64),
                ("launches", ctypes.c_uint64), ("elements", ctypes.c_uint64), ("p50_ms", ctypes.c_double),
                ("p99_ms", ctypes.c_double), ("mean_ms", ctypes.c_double), ("max_ms", ctypes.c_double),
                ("first_submit_to_last_done_ms", ctypes.c_double)]


class ZodaTiming(ctypes.Structure):
    _fields_ = [("h2d_ms", ctypes.c_float), ("kernel_ms", ctypes.c_float),
                ("d2h_ms", ctypes.c_float), ("total_ms", ctypes.c_float),
                ("h2d_bytes", ctypes.c_uint64), ("d2h_bytes", ctypes.c_uint64)]


class ZodaPlan(ctypes.Structure):
    """Per-side launch plan (include/zoda_b200.h, zoda_plan)."""
    _fields_ = [("impl", ctypes.c_int32), ("sched", ctypes.c_int32), ("l2_promo", ctypes.c_int32),
                ("blocked", ctypes.c_int32), ("stagger", ctypes.c_int32), ("radix", ctypes.c_int32),
                ("ms", ctypes.c_float), ("ctas", ctypes.c_int32)]
    KEYS = ("impl", "sched", "l2_promo", "blocked", "stagger", "radix", "ms", "ctas")
    DEFAULTS = {"radix": 16, "ctas": 0}

    def to_dict(self) -> dict:
        return {k: (round(float(getattr(self, k)), 5) if k == "ms" else int(getattr(self, k))) for k in self.KEYS}

    @classmethod
    def from_dict(cls, d: dict) -> "ZodaPlan":
        return cls(*[d.get(k, cls.DEFAULTS.get(k, 0)) for k in cls.KEYS])


def load(path: str = LIB_PATH):
    """Load the library and declare every exported signature. Raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise FileNotFoundError(f"{path} is not built; run `make -C {HERE}`")
    L = ctypes.CDLL(path)
    u32p = ctypes.POINTER(ctypes.c_uint32)
    vp = ctypes.c_void_p
    L.cuda_ntt.restype = ctypes.c_int
    L.cuda_ntt.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    L.cuda_intt.restype = ctypes.c_int
    L.cuda_intt.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint32]
    L.cuda_host_alloc.restype = vp
    L.cuda_host_alloc.argtypes = [ctypes.c_size_t]
    L.cuda_host_free.restype = None
    L.cuda_host_free.argtypes = [vp]
    L.zoda_status_string.restype = ctypes.c_char_p
    L.zoda_status_string.argtypes = [ctypes.c_int]
    L.zoda_last_error.restype = ctypes.c_char_p
    L.zoda_last_error.argtypes = []
    L.zoda_ctx_create.restype = ctypes.c_int
    L.zoda_ctx_create.argtypes = [ctypes.c_int, ctypes.POINTER(vp)]
    L.zoda_ctx_destroy.restype = None
    L.zoda_ctx_destroy.argtypes = [vp]
    L.zoda_max_side.restype = ctypes.c_uint32
    L.zoda_max_side.argtypes = []
    L.zoda_extend_device.restype = ctypes.c_int
    L.zoda_extend_device.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint64, vp]
    L.zoda_ctx_set_impl.restype = ctypes.c_int
    L.zoda_ctx_set_impl.argtypes = [vp, ctypes.c_int]
    L.zoda_ctx_check.restype = ctypes.c_int
    L.zoda_ctx_check.argtypes = [vp]
    L.zoda_selftest_bounded_wait.restype = ctypes.c_int
    L.zoda_selftest_bounded_wait.argtypes = [vp, vp]
    L.zoda_batch_create.restype = ctypes.c_int
    L.zoda_batch_create.argtypes = [vp, ctypes.POINTER(ZodaSquare), ctypes.c_uint32, ctypes.POINTER(vp)]
    L.zoda_batch_run.restype = ctypes.c_int
    L.zoda_batch_run.argtypes = [vp, vp]
    L.zoda_batch_elements.restype = ctypes.c_uint64
    L.zoda_batch_elements.argtypes = [vp]
    L.zoda_batch_destroy.restype = None
    L.zoda_batch_destroy.argtypes = [vp]
    L.zoda_server_create.restype = ctypes.c_int
    L.zoda_server_create.argtypes = [vp, ctypes.POINTER(ZodaServerConfig), ctypes.POINTER(vp)]
    L.zoda_server_submit.restype = ctypes.c_int
    L.zoda_server_submit.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64)]
    L.zoda_server_wait.restype = ctypes.c_int
    L.zoda_server_wait.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint32, ctypes.POINTER(ZodaRequestInfo)]
    L.zoda_server_release.restype = ctypes.c_int
    L.zoda_server_release.argtypes = [vp, ctypes.c_uint64]
    L.zoda_server_cancel.restype = ctypes.c_int
    L.zoda_server_cancel.argtypes = [vp, ctypes.c_uint64]
    L.zoda_server_get_stats.restype = ctypes.c_int
    L.zoda_server_get_stats.argtypes = [vp, ctypes.POINTER(ZodaServerStats)]
    L.zoda_server_destroy.restype = None
    L.zoda_server_destroy.argtypes = [vp]
    L.zoda_encode_device.restype = ctypes.c_int
    L.zoda_encode_device.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, vp]
    L.zoda_recover_device.restype = ctypes.c_int
    L.zoda_recover_device.argtypes = [vp, vp, u32p, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, vp,
                                      ctypes.POINTER(ctypes.c_uint64), vp]
    L.zoda_autotune.restype = ctypes.c_int
    L.zoda_autotune.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_uint32,
                                ctypes.POINTER(ZodaPlan)]
    L.zoda_plan_get.restype = ctypes.c_int
    L.zoda_plan_get.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(ZodaPlan)]
    L.zoda_plan_set.restype = ctypes.c_int
    L.zoda_plan_set.argtypes = [vp, ctypes.c_uint32, ctypes.POINTER(ZodaPlan)]
    L.zoda_plan_clear.restype = None
    L.zoda_plan_clear.argtypes = [vp]
    L.zoda_data_root_host.restype = ctypes.c_int
    L.zoda_data_root_host.argtypes = [vp, ctypes.c_uint64, ctypes.c_uint64, ctypes.c_char_p]
    L.zoda_rlc_coefficients_device.restype = ctypes.c_int
    L.zoda_rlc_coefficients_device.argtypes = [vp, ctypes.c_char_p, ctypes.c_size_t, ctypes.c_uint64, vp, vp]
    L.zoda_rlc_rows_device.restype = ctypes.c_int
    L.zoda_rlc_rows_device.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint64, vp, vp, vp]
    L.zoda_rlc_check_device.restype = ctypes.c_int
    L.zoda_rlc_check_device.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_uint64, vp,
                                        ctypes.POINTER(ctypes.c_uint64), vp]
    L.zoda_ntt_device_noalloc.restype = ctypes.c_int
    L.zoda_ntt_device_noalloc.argtypes = [vp, vp, ctypes.c_uint32, ctypes.c_uint32, ctypes.c_int, vp]
    L.zoda_ctx_inject_fault.restype = ctypes.c_int
    L.zoda_ctx_inject_fault.argtypes = [vp, ctypes.c_uint32, ctypes.c_uint32]
    L.zoda_extend_host.restype = ctypes.c_int
    L.zoda_extend_host.argtypes = [vp, vp, vp, ctypes.c_uint32, ctypes.c_uint64, ctypes.POINTER(ZodaTiming)]
    del u32p
    _lib = L
    return L


def _check(status: int, where: str):
    if status != ZODA_OK:
        detail = load().zoda_last_error().decode(errors="replace")
        raise ZodaError(status, where, detail)


def _addr(buf) -> int:
    """Address of a torch tensor, numpy array or raw int pointer."""
    if isinstance(buf, int):
        return buf
    if hasattr(buf, "data_ptr"):
        return buf.data_ptr()
    if hasattr(buf, "ctypes"):
        return buf.ctypes.data
    raise TypeError(f"cannot take the address of {type(buf)}")


class Context:
    """A device context: twiddle tables resident in HBM, a stream, cached buffers."""

    def __init__(self, device: int = 0):
        L = load()
        h = ctypes.c_void_p()
        _check(L.zoda_ctx_create(device, ctypes.byref(h)), "zoda_ctx_create")
        self._h = h
        self.device = device

    @property
    def handle(self):
        return self._h

    def close(self):
        if self._h:
            load().zoda_ctx_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def extend(self, d_in, d_out, k: int, cols: int, stream=None):
        """Fused extension on device buffers: d_in [k][cols] -> d_out [2k][cols] (row-major u32).
        `stream` is a torch.cuda.Stream, a raw cudaStream_t int, or None for torch's current
        stream (so torch events and later torch work order correctly against the kernel)."""
        if stream is None:
            import torch
            stream = torch.cuda.current_stream()
        s = stream if isinstance(stream, int) else stream.cuda_stream
        _check(load().zoda_extend_device(self._h, _addr(d_in), _addr(d_out), k, cols, s or None),
               "zoda_extend_device")

    def encode(self, d_in, d_out, k: int, n: int, cols: int, stream=None):
        """Encode of any shape (src/benchmarks/utils.rs:100-146): d_in [k][cols] ->
        d_out [k+n][cols], rows 0..k+n-1 of the evaluation over next_pow2(k+n) points."""
        _check(load().zoda_encode_device(self._h, _addr(d_in), _addr(d_out), k, n, cols, _stream_handle(stream)),
               "zoda_encode_device")

    def recover(self, d_code, known_rows, k: int, cols: int, d_data, check: bool = False, stream=None):
        """k-of-2k erasure recovery: d_code [2k][cols] with only `known_rows` valid ->
        d_data [k][cols]. With check=True returns the number of inconsistent
        coefficients (0 when the known rows are one codeword) and synchronizes."""
        rows = sorted(set(int(r) for r in known_rows))
        arr = (ctypes.c_uint32 * max(1, len(rows)))(*rows)
        mm = ctypes.c_uint64(0)
        _check(load().zoda_recover_device(self._h, _addr(d_code), arr, len(rows), k, cols, _addr(d_data),
                                          ctypes.byref(mm) if check else None, _stream_handle(stream)),
               "zoda_recover_device")
        return int(mm.value) if check else None

    def rlc_coefficients(self, root: str, ncols: int, d_coeff, stream=None):
        """src/zoda/rlc.rs:48-65 on the device: d_coeff [ncols][4] u32 from the data root's hex string."""
        b = root.encode()
        _check(load().zoda_rlc_coefficients_device(self._h, b, len(b), ncols, _addr(d_coeff),
                                                   _stream_handle(stream)), "zoda_rlc_coefficients_device")

    def rlc_rows(self, d_rows, rows: int, cols: int, d_coeff, d_out, stream=None):
        """src/zoda/rlc.rs:32-40 for every row: d_out [rows][4]."""
        _check(load().zoda_rlc_rows_device(self._h, _addr(d_rows), rows, cols, _addr(d_coeff), _addr(d_out),
                                           _stream_handle(stream)), "zoda_rlc_rows_device")

    def rlc_check(self, d_data, d_code, k: int, n: int, cols: int, d_coeff, stream=None) -> int:
        """RLC check of every encoded row (src/benchmarks/utils.rs:225-272); returns the
        number of mismatching (row, limb) pairs, 0 when the encoding passes."""
        mm = ctypes.c_uint64(0)
        _check(load().zoda_rlc_check_device(self._h, _addr(d_data), _addr(d_code), k, n, cols, _addr(d_coeff),
                                            ctypes.byref(mm), _stream_handle(stream)), "zoda_rlc_check_device")
        return int(mm.value)

    def autotune(self, side_min: int, side_max: int, cols: int = 0, reps: int = 5) -> dict:
        """Tune every power-of-two side in [side_min, side_max]; returns {side: plan dict}
        and installs the chosen plans on this context."""
        arr = (ZodaPlan * 13)()
        _check(load().zoda_autotune(self._h, side_min, side_max, cols, reps, arr), "zoda_autotune")
        out, s = {}, side_min
        while s <= side_max:
            out[s] = arr[s.bit_length() - 1].to_dict()
            s *= 2
        return out

    def plan_get(self, side: int):
        """The side's installed plan as a dict, or None when it has none."""
        p = ZodaPlan()
        st = load().zoda_plan_get(self._h, side, ctypes.byref(p))
        if st == 8:  # ZODA_ERR_STATE: no plan
            return None
        _check(st, "zoda_plan_get")
        return p.to_dict()

    def plan_set(self, side: int, plan: dict):
        p = ZodaPlan.from_dict(plan)
        _check(load().zoda_plan_set(self._h, side, ctypes.byref(p)), "zoda_plan_set")

    def plan_clear(self):
        load().zoda_plan_clear(self._h)

    def save_plans(self, path: str):
        """Write every installed plan as JSON {side: plan} (a tuning cache)."""
        plans = {}
        for ls in range(13):
            p = self.plan_get(1 << ls)
            if p is not None:
                plans[str(1 << ls)] = p
        with open(path, "w") as f:
            json.dump(plans, f, indent=1, sort_keys=True)

    def load_plans(self, path: str):
        with open(path) as f:
            plans = json.load(f)
        for side, p in plans.items():
            self.plan_set(int(side), p)

    def set_impl(self, impl: int):
        """0 = automatic, 1 = direct-load kernel, 2 = TMA-staged kernel, 3 = four-step passes."""
        _check(load().zoda_ctx_set_impl(self._h, impl), "zoda_ctx_set_impl")

    def check(self):
        """Raise if a kernel on this context gave up a bounded wait (synchronizes)."""
        _check(load().zoda_ctx_check(self._h), "zoda_ctx_check")

    def selftest_bounded_wait(self, stream=None):
        """Run a kernel whose barrier wait nothing completes; the next check() raises
        ZODA_ERR_TIMEOUT (and clears the flag)."""
        _check(load().zoda_selftest_bounded_wait(self._h, _stream_handle(stream)), "zoda_selftest_bounded_wait")

    def inject_fault(self, site: int, after: int = 0):
        """Arm a fault site (zoda_ctx_inject_fault): 1 = a column-chunk launch of
        extend_host, failing after `after` chunks; 2 = a pipelined four-step launch
        whose dependency waits run out; 0 disarms."""
        _check(load().zoda_ctx_inject_fault(self._h, site, after), "zoda_ctx_inject_fault")

    def extend_host(self, h_in, h_out, k: int, cols: int) -> ZodaTiming:
        t = ZodaTiming()
        _check(load().zoda_extend_host(self._h, _addr(h_in), _addr(h_out), k, cols, ctypes.byref(t)),
               "zoda_extend_host")
        return t


def data_root(rows) -> str:
    """compute_data_root (src/benchmarks/utils.rs:51-59) of a host row-major u32 array
    (numpy), computed by the library's host SHA-256."""
    import numpy as np
    a = np.ascontiguousarray(rows, dtype=np.uint32)
    out = ctypes.create_string_buffer(65)
    nrows = a.shape[0] if a.ndim > 1 else 1
    _check(load().zoda_data_root_host(a.ctypes.data, nrows, a.size // max(1, nrows), out), "zoda_data_root_host")
    return out.value.decode()


def _stream_handle(stream):
    if stream is None:
        import torch
        stream = torch.cuda.current_stream()
    s = stream if isinstance(stream, int) else stream.cuda_stream
    return s or None


class Batch:
    """Many squares of mixed sides (32..2048) encoded by one persistent,
    graph-captured launch (zoda_batch_create / zoda_batch_run)."""

    def __init__(self, ctx: Context, squares):
        """squares: iterable of (d_in, d_out, k, cols) on the context's device."""
        sq = list(squares)
        arr = (ZodaSquare * max(1, len(sq)))()
        for i, (a, b, k, cols) in enumerate(sq):
            arr[i] = ZodaSquare(_addr(a), _addr(b), k, 0, cols)
        h = ctypes.c_void_p()
        _check(load().zoda_batch_create(ctx.handle, arr, len(sq), ctypes.byref(h)), "zoda_batch_create")
        self._h = h
        self._keep = sq  # the buffers must outlive the batch

    @property
    def elements(self) -> int:
        return int(load().zoda_batch_elements(self._h))

    def run(self, stream=None):
        _check(load().zoda_batch_run(self._h, _stream_handle(stream)), "zoda_batch_run")

    def close(self):
        if self._h:
            load().zoda_batch_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


_cudart = None


def device_copy(dst, src, nbytes: int):
    """cudaMemcpy (device to device) between raw addresses or tensors; used to read
    outputs that live in a server's arena."""
    global _cudart
    if _cudart is None:
        _cudart = ctypes.CDLL("libcudart.so.12")
        _cudart.cudaMemcpy.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_size_t, ctypes.c_int]
        _cudart.cudaMemcpy.restype = ctypes.c_int
    err = _cudart.cudaMemcpy(_addr(dst), _addr(src), nbytes, 3)
    if err != 0:
        raise RuntimeError(f"cudaMemcpy failed with {err}")


class Server:
    """Serving loop with continuous batching (zoda_server_*): submit squares as they
    arrive, wait for each, read its output from the server's arena, release it."""

    def __init__(self, ctx: Context, budget_bytes: int = 0, max_inflight: int = 0, max_batch: int = 0):
        cfg = ZodaServerConfig(budget_bytes, max_inflight, max_batch)
        h = ctypes.c_void_p()
        _check(load().zoda_server_create(ctx.handle, ctypes.byref(cfg), ctypes.byref(h)), "zoda_server_create")
        self._h = h

    def submit(self, d_in, k: int, cols: int) -> int:
        t = ctypes.c_uint64()
        _check(load().zoda_server_submit(self._h, _addr(d_in), k, cols, ctypes.byref(t)), "zoda_server_submit")
        return t.value

    def wait(self, ticket: int, timeout_ms: int = 60000) -> ZodaRequestInfo:
        info = ZodaRequestInfo()
        _check(load().zoda_server_wait(self._h, ticket, timeout_ms, ctypes.byref(info)), "zoda_server_wait")
        return info

    def release(self, ticket: int):
        _check(load().zoda_server_release(self._h, ticket), "zoda_server_release")

    def cancel(self, ticket: int):
        _check(load().zoda_server_cancel(self._h, ticket), "zoda_server_cancel")

    def stats(self) -> ZodaServerStats:
        st = ZodaServerStats()
        _check(load().zoda_server_get_stats(self._h, ctypes.byref(st)), "zoda_server_get_stats")
        return st

    def close(self):
        if self._h:
            load().zoda_server_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def max_side() -> int:
    return int(load().zoda_max_side())


# ---- mirror of src/ntt/cuda.rs ----------------------------------------------

def cuda_available() -> bool:
    """src/ntt/cuda.rs:25-29 through the CUDA runtime the library links."""
    try:
        import torch
        return torch.cuda.is_available() and torch.cuda.device_count() > 0
    except Exception:
        return False


def _run(values, n: int, stride: int, fn, name: str, roots=None):
    """src/ntt/cuda.rs:99-119: argument checks, roots_of_unity(n), the FFI call."""
    import numpy as np
    assert n > 0 and (n & (n - 1)) == 0, "NTT size must be power of 2"
    assert stride >= n, "stride must be at least n"
    size = values.size if hasattr(values, "size") and not callable(values.size) else values.numel()
    assert stride > 0 and size % stride == 0, "values must be whole polynomials of stride elements"
    polys = size // stride
    if roots is None:
        roots = _roots_of_unity(n)
    roots = np.ascontiguousarray(roots, dtype=np.uint32)
    err = fn(_addr(values), roots.ctypes.data, n, polys, stride)
    if err != 0:
        raise RuntimeError(f"{name} failed with CUDA error {err}")


def _roots_of_unity(n: int):
    """[w^0 .. w^(n-1)] for w = 31^((p-1)/n), the roots src/ntt/cpu.rs:96-110 derives."""
    import numpy as np
    w = pow(31, (P - 1) // n, P)
    out = np.empty(n, dtype=np.uint32)
    cur = 1
    for i in range(n):
        out[i] = cur
        cur = cur * w % P
    return out


def ntt_cuda(values, n: int, stride: int, roots=None):
    """src/ntt/cuda.rs:124-126: forward NTT on the GPU, in place, host buffer."""
    _run(values, n, stride, load().cuda_ntt, "cuda_ntt", roots)


def intt_cuda(values, n: int, stride: int, roots=None):
    """src/ntt/cuda.rs:129-131: inverse NTT on the GPU, in place, host buffer."""
    _run(values, n, stride, load().cuda_intt, "cuda_intt", roots)


class PinnedSquare:
    """src/ntt/cuda.rs:34-97: `cols` polynomials of `rows` canonical u32 each, column-major,
    in pinned host memory from cuda_host_alloc; element (row, col) at col*rows + row."""

    def __init__(self, rows: int, cols: int):
        import numpy as np
        count = max(rows * cols, 1)
        ptr = load().cuda_host_alloc(count)
        if not ptr:
            raise MemoryError(f"cudaHostAlloc of {count} u32 failed")
        self._ptr = ptr
        self.rows, self.cols = rows, cols
        buf = (ctypes.c_uint32 * count).from_address(ptr)
        self.array = np.frombuffer(buf, dtype=np.uint32, count=rows * cols)
        self.array[:] = 0

    def set(self, row, col, value):
        self.array[col * self.rows + row] = value

    def get(self, row, col):
        return int(self.array[col * self.rows + row])

    def column(self, col):
        return self.array[col * self.rows:(col + 1) * self.rows]

    def row(self, row):
        return self.array[row::self.rows][:self.cols]

    @property
    def size(self):
        return self.rows * self.cols

    @property
    def ctypes(self):
        return self.array.ctypes

    def free(self):
        if self._ptr:
            self.array = None
            load().cuda_host_free(self._ptr)
            self._ptr = None

    def __del__(self):
        try:
            self.free()
        except Exception:
            pass
