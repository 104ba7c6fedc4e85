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

    python -m dftbaby_b200.gemm_bench --ozaki --m 4146 --n 4146 --k 4146 [--nmod 16]

times the FP64 product A B of the int8 tensor-core emulation (ozaki.matmul: residues, nmod int8 GEMMs,
reconstruction) against cuBLAS DGEMM on the same matrices and reports the MMA kernel's rate against the
dense int8 peak (2x the measured BF16 figure).
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
    ap.add_argument("--wide", action="store_true", help="split mode on 128 x 256 tiles")
    ap.add_argument("--ozaki", action="store_true")
    ap.add_argument("--nmod", type=int, default=16)
    ap.add_argument("--phases", action="store_true", help="with --ozaki: per-kernel device time (CUPTI)")
    a = ap.parse_args()
    native.load()
    dev = torch.device("cuda", 0)
    if a.ozaki:
        return ozaki_main(a, dev)
    g = torch.Generator(device="cpu").manual_seed(0)
    A = torch.randn(a.m, a.k, generator=g, dtype=torch.float32).to(dev)
    B = torch.randn(a.n, a.k, generator=g, dtype=torch.float32).to(dev)
    pa, pb = tcgemm.split(A), tcgemm.split(B)
    C = tcgemm.Pair(a.m, a.n, dev)
    kw = dict(K=a.k, out_pair=C, wide=a.wide)
    if a.epilogue == "f32":
        # FP32 output, K split over several CTAs when the output has fewer tiles than SMs
        kw = dict(K=a.k, alpha=0.25, out=torch.empty((a.m, a.n), dtype=torch.float32, device=dev), wide=a.wide)
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
    print(json.dumps({"shape": [a.m, a.n, a.k], "epilogue": a.epilogue, "segments": 3, "wide": a.wide, "ms": ms,
                      "tflops": tf, "peak_bf16_tflops": peak,
                      "frac": tf / peak}))


def _peaks():
    peak_file = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "MEASURED_PEAKS.json")
    return json.load(open(peak_file)) if os.path.exists(peak_file) else {}


def ozaki_main(a, dev):
    from . import ozaki
    g = torch.Generator(device="cpu").manual_seed(0)
    A = torch.randn(a.m, a.k, generator=g, dtype=torch.float64).to(dev)
    B = torch.randn(a.k, a.n, generator=g, dtype=torch.float64).to(dev)
    C = torch.empty(a.m, a.n, dtype=torch.float64, device=dev)

    def timed(fn):
        for _ in range(a.warmup):
            fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        for _ in range(a.reps):
            fn()
        e1.record()
        e1.synchronize()
        return e0.elapsed_time(e1) / a.reps

    ms = timed(lambda: ozaki.matmul(A, B, out=C, nmod=a.nmod))
    ozaki.check_errors(dev)
    ms_dgemm = timed(lambda: torch.matmul(A, B, out=C))
    ref = A @ B
    err = ((ozaki.matmul(A, B, nmod=a.nmod) - ref).abs().max() / ref.abs().max()).item()
    flops = 2.0 * a.m * a.n * a.k
    int8_ops = flops * a.nmod  # executed on the tensor cores (unpadded shape)
    peak_i8 = 2.0 * _peaks().get("bf16_tflops", 1590.0)
    out = {"shape": [a.m, a.n, a.k], "nmod": a.nmod, "ms": ms, "fp64_equivalent_tflops": flops / ms / 1e9,
           "ms_cublas_dgemm": ms_dgemm, "dgemm_tflops": flops / ms_dgemm / 1e9, "speedup_vs_dgemm": ms_dgemm / ms,
           "int8_tops_whole_call": int8_ops / ms / 1e9, "peak_int8_tops": peak_i8, "max_rel_err_vs_dgemm": err}
    if a.phases:
        # device time per kernel of a.reps calls (CUDA activity records through torch.profiler)
        from torch.profiler import ProfilerActivity, profile
        with profile(activities=[ProfilerActivity.CUDA]) as prof:
            for _ in range(a.reps):
                ozaki.matmul(A, B, out=C, nmod=a.nmod)
            torch.cuda.synchronize()
        out["kernel_ms_per_call"] = {k.key.split("(")[0]: k.device_time_total / 1e3 / a.reps
                                     for k in prof.key_averages()
                                     if k.device_type.name == "CUDA" and k.device_time_total > 0}
    print(json.dumps(out))


if __name__ == "__main__":
    main()
