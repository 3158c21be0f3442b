"""Measured dense-GEMM peaks that the DCT kernels are judged against.

The roofline of a tensor-core kernel needs the peak of its own arithmetic:
the precision form's DCT runs split-TF32 products, the FP64 form's
fallback contraction FP64 (DMMA) products.  This measures both as the
library GEMM rate on square operands (torch.matmul -> cuBLAS), burst
(best of 10 launches) and sustained (back to back for ~3 s), with CUDA
events on one GPU; no clock or power setting is touched.

    python -m pllcart3d_b200.peaks [--out FILE.json]
"""

from __future__ import annotations

import argparse
import json
import time


def _rate(dtype, n, tf32, seconds):
    import torch

    torch.backends.cuda.matmul.allow_tf32 = tf32
    a = torch.randn(n, n, device="cuda", dtype=dtype)
    b = torch.randn(n, n, device="cuda", dtype=dtype)
    c = torch.empty(n, n, device="cuda", dtype=dtype)
    flops = 2.0 * n * n * n
    for _ in range(3):
        torch.matmul(a, b, out=c)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(10):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b, out=c)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1))
    burst = flops / (best / 1e3) / 1e12
    # sustained: back to back for ~seconds
    reps = max(1, int(seconds / (best / 1e3)))
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(reps):
        torch.matmul(a, b, out=c)
    e1.record()
    torch.cuda.synchronize()
    sustained = flops * reps / (e0.elapsed_time(e1) / 1e3) / 1e12
    torch.backends.cuda.matmul.allow_tf32 = False
    return {"n": n, "burst_tflops": burst, "sustained_tflops": sustained, "reps": reps}


def measure(seconds: float = 3.0) -> dict:
    import torch

    out = {"gpu": torch.cuda.get_device_name(0), "how": "torch.matmul (cuBLAS) on n x n operands, CUDA events; "
           "burst = best of 10, sustained = back to back", "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}
    out["fp64"] = _rate(torch.float64, 8192, False, seconds)
    out["tf32"] = _rate(torch.float32, 8192, True, seconds)
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=None)
    ap.add_argument("--seconds", type=float, default=3.0)
    args = ap.parse_args(argv)
    res = measure(args.seconds)
    print(json.dumps(res), flush=True)
    if args.out:
        with open(args.out, "w") as f:
            json.dump(res, f, indent=1)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
