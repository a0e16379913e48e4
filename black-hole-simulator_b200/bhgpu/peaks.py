"""FP64 / FP32 multiply-add throughput of the current GPU (bh_peak_fma).

The stencil kernels of this library are bound by their FP64 (or, in the
mixed variant, FP32) instruction throughput rather than by HBM; these
figures are the denominators of that roofline.
"""
from __future__ import annotations

import ctypes as C

import torch

from ._lib import BH_FP64, BH_MIXED, check, lib

lib.bh_peak_fma.argtypes = [C.c_int32, C.c_int32, C.c_void_p, C.c_int64, C.POINTER(C.c_int64), C.c_void_p]
lib.bh_peak_fma.restype = C.c_int


def fma_peak(precision: str = "fp64", iters: int = 4096, reps: int = 5) -> float:
    """Measured multiply-add throughput in TFLOP/s ('fp64' or 'fp32')."""
    dev = torch.cuda.current_device()
    sms = torch.cuda.get_device_properties(dev).multi_processor_count
    n = sms * 8 * 256
    dt = torch.float64 if precision == "fp64" else torch.float32
    code = BH_FP64 if precision == "fp64" else BH_MIXED
    out = torch.empty(n, dtype=dt, device="cuda")
    flops = C.c_int64()
    s = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    check(lib.bh_peak_fma(code, iters, C.c_void_p(out.data_ptr()), n, C.byref(flops), s), "bh_peak_fma")
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    best = 0.0
    for _ in range(reps):
        a.record()
        check(lib.bh_peak_fma(code, iters, C.c_void_p(out.data_ptr()), n, C.byref(flops), s), "bh_peak_fma")
        b.record()
        torch.cuda.synchronize()
        best = max(best, flops.value / (a.elapsed_time(b) * 1e-3) / 1e12)
    return best
