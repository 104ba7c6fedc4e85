"""Microbenchmark of the transition-charge entry point (the source of the tc_tile_kernel profile).

    python -m dftbaby_b200.tc_bench NAT NOCC NVIRT [REPS]

Calls dftb_trans_charges for the occupied-virtual block only on random coefficients and overlap (a quarter
of the atoms hydrogen with one orbital, the rest carbon with four), times REPS calls with CUDA events after
one warm-up call and prints the q_ov bytes written per second of the whole call (the two S.C products
included), then the device time of each kernel of one more call (CUDA activity records) with the tile
kernel's own rate.  ``1104 1225 1225`` is the size of the 1104-atom benchmark's window; ``600 300 300 1`` is the
small case profiled under ncu.
"""
import sys

import numpy as np
import torch

from . import native


def main(argv=None):
    argv = sys.argv[1:] if argv is None else argv
    nat, no, nv = int(argv[0]), int(argv[1]), int(argv[2])
    reps = int(argv[3]) if len(argv) > 3 else 5
    L = native.load()
    rng = np.random.default_rng(0)
    opa = np.where(rng.random(nat) < 0.25, 1, 4).astype(np.int32)
    norb = int(opa.sum())
    dev = torch.device("cuda")
    g = torch.Generator(device="cpu").manual_seed(0)
    Co = torch.randn(norb, no, generator=g, dtype=torch.float64).to(dev)
    Cv = torch.randn(norb, nv, generator=g, dtype=torch.float64).to(dev)
    S = torch.randn(norb, norb, generator=g, dtype=torch.float64).to(dev)
    S = 0.5 * (S + S.T)
    opa_d = torch.as_tensor(opa, device=dev)
    q = torch.empty(nat, no, nv, dtype=torch.float64, device=dev)
    nb = L.dftb_trans_charges_workspace_size(norb, no, nv)
    ws = torch.empty(nb, dtype=torch.uint8, device=dev)
    P = native.ptr

    def call():
        native.call("dftb_trans_charges", norb, nat, no, nv, P(Co), P(Cv), P(S), P(opa_d), None, P(q), None, P(ws), nb,
                    native.stream())

    call()
    torch.cuda.synchronize()
    ts = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        call()
        e1.record()
        e1.synchronize()
        ts.append(e0.elapsed_time(e1))
    gb = 8.0 * nat * no * nv / 1e9
    print("nat %d norb %d window %dx%d: q_ov %.2f GB, whole call %.3f ms (min %.3f) -> %.0f GB/s of q_ov writes" % (
        nat, norb, no, nv, gb, float(np.median(ts)), min(ts), gb / (min(ts) / 1e3)))
    # device time per kernel of one call (CUDA activity records): the tile kernel alone against the q_ov bytes
    from torch.profiler import ProfilerActivity, profile
    with profile(activities=[ProfilerActivity.CUDA]) as prof:
        call()
        torch.cuda.synchronize()
    for k in prof.key_averages():
        if k.device_type.name == "CUDA" and k.device_time_total > 0:
            ms = k.device_time_total / 1e3
            extra = " -> %.0f GB/s of q_ov writes" % (gb / (ms / 1e3)) if "tc_tile" in k.key else ""
            name = k.key.replace("(anonymous namespace)::", "").split("(")[0] or k.key
            print("  %-60s %8.3f ms%s" % (name[:60], ms, extra))


if __name__ == "__main__":
    main()
