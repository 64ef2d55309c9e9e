"""Measure the FP64 denominator of the roofline on the current GPU.

MEASURED_PEAKS.json holds HBM copy bandwidth and bf16 GEMM throughput only;
the DQMC path computes in FP64, so its compute roofline is the FP64 DGEMM
throughput of the same GPU (cuBLAS through torch.matmul on float64, which runs
on the FP64 tensor pipe).  Writes profiles/fp64_peak_b200.json.

    python -m z2_gauge_zfy_b200.peaks
"""
import json
import os
import time

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def measure(n: int = 8192, reps: int = 10):
    import torch
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize()
    best = float("inf")
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    flops = 2.0 * n ** 3
    return {"dgemm_tflops": flops / best / 1e12, "n": n, "best_s": best,
            "how": "torch.matmul float64 n^3 (2 n^3 flops), best of %d, CUDA events" % reps,
            "gpu": torch.cuda.get_device_name(0),
            "when": time.strftime("%Y-%m-%dT%H:%M:%SZ", time.gmtime())}


if __name__ == "__main__":
    d = measure()
    out = os.path.join(ROOT, "profiles", "fp64_peak_b200.json")
    os.makedirs(os.path.dirname(out), exist_ok=True)
    with open(out, "w") as f:
        json.dump(d, f, indent=1)
    print(json.dumps(d))
