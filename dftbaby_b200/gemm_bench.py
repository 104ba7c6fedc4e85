"""Microbenchmark of the split-precision tensor-core GEMM at a given shape.

    python -m dftbaby_b200.gemm_bench --m 1225 --n 8292 --k 8292 [--reps 20] [--epilogue pair|gpt]

Times alpha * A B^T (A: m x k, B: n x k, BF16 hi/lo pairs, three products
accumulated in FP32) with CUDA events after warm-up and prints TFLOP/s against
the BF16 peak in MEASURED_PEAKS.json.  The default shape is the largest
exchange contraction of the 1104-atom benchmark (P^T = Ybar^T N).  With
``--epilogue gpt`` the result is multiplied elementwise by an FP32 matrix G and
stored as a hi/lo pair both row-major and transposed, as in the exchange
contraction N = X_o W o G_lr (``--m 8292 --n 4146 --k 1225`` at that benchmark);
``--epilogue f32`` stores FP32 (the final K contraction, ``--m 1225 --n 1225 --k 8292``).
"""
import argparse
import json
import os

import torch

from . import native, tcgemm


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--m", type=int, default=1225)
    ap.add_argument("--n", type=int, default=8292)
    ap.add_argument("--k", type=int, default=8292)
    ap.add_argument("--reps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--epilogue", choices=["pair", "gpt", "f32"], default="pair")
    a = ap.parse_args()
    native.load()
    dev = torch.device("cuda", 0)
    g = torch.Generator(device="cpu").manual_seed(0)
    A = torch.randn(a.m, a.k, generator=g, dtype=torch.float32).to(dev)
    B = torch.randn(a.n, a.k, generator=g, dtype=torch.float32).to(dev)
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C = tcgemm.Pair(a.m, a.n, dev)
    kw = dict(K=a.k, out_pair=C)
    if a.epilogue == "f32":
        # FP32 output, K split over several CTAs when the output has fewer tiles than SMs
        kw = dict(K=a.k, alpha=0.25, out=torch.empty((a.m, a.n), dtype=torch.float32, device=dev))
    if a.epilogue == "gpt":
        kw.update(G=torch.rand(a.m, a.n, generator=g, dtype=torch.float32).to(dev),
                  out_pair_t=tcgemm.Pair(a.n, a.m, dev))
    for _ in range(a.warmup):
        tcgemm.gemm(pa, pb, **kw)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(a.reps):
        tcgemm.gemm(pa, pb, **kw)
    e1.record()
    e1.synchronize()
    tcgemm.check_errors(dev)
    ms = e0.elapsed_time(e1) / a.reps
    flops = 2.0 * a.m * a.n * a.k * 3
    peak_file = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    peak = json.load(open(peak_file)).get("bf16_tflops", 1637.5) if os.path.exists(peak_file) else 1590.0
    tf = flops / (ms / 1e3) / 1e12
    print(json.dumps({"shape": [a.m, a.n, a.k], "epilogue": a.epilogue, "segments": 3, "ms": ms, "tflops": tf, "peak_bf16_tflops": peak,
                      "frac": tf / peak}))


if __name__ == "__main__":
    main()
