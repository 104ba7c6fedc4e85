"""The allocation-free transition-charge entry point against the workspace one.

dftb_trans_charges_noalloc serves callers that cannot allocate device memory
(a host that has reserved the GPU's memory in its own pool, or a binding that
only receives device pointers): it keeps its scratch in a fixed device array
instead of a caller workspace.  Its results must equal dftb_trans_charges on
the same inputs, also on a second call right after the first (the shared
scratch keeps the previous call's contents), and requests larger than the
array must be refused without launching anything.

This file is collected last so that a run stopping at the first failure has
already run every other test.
"""
import numpy as np
import pytest
import torch

from dftbaby_b200 import geometry, native
from oracle import dftb_oracle as O

pytestmark = pytest.mark.gpu

TOL = 1e-13  # the same tolerance the transition-charge parity test uses


def _inputs(n_carbons, seed, dev):
    al = geometry.polyene(n_carbons, sigma=0.02, seed=seed)
    o = O.DFTB2(al, long_range_correction=0)
    o.setGeometry(al)
    o.getEnergy()
    no = int(np.sum(o.f > 0.1))
    t = lambda a: torch.as_tensor(np.ascontiguousarray(a), device=dev)
    return dict(nat=len(al), norb=o.dim, no=no, nv=o.dim - no, Co=t(o.orbs[:, :no]), Cv=t(o.orbs[:, no:]),
                S=t(o.S), opa=torch.tensor(o.orbsPerAtom, dtype=torch.int32, device=dev))


def _outputs(x, dev):
    e = lambda *shape: torch.full(shape, np.nan, dtype=torch.float64, device=dev)
    return e(x["nat"], x["no"], x["no"]), e(x["nat"], x["no"], x["nv"]), e(x["nat"], x["nv"], x["nv"])


def _with_workspace(x, dev):
    L = native.load()
    out = _outputs(x, dev)
    nbytes = L.dftb_trans_charges_workspace_size(x["norb"], x["no"], x["nv"])
    ws = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    P = native.ptr
    native.call("dftb_trans_charges", x["norb"], x["nat"], x["no"], x["nv"], P(x["Co"]), P(x["Cv"]), P(x["S"]),
                P(x["opa"]), P(out[0]), P(out[1]), P(out[2]), P(ws), nbytes, native.stream())
    torch.cuda.synchronize()
    return [a.cpu().numpy() for a in out]


def _without_allocation(x, dev):
    out = _outputs(x, dev)
    P = native.ptr
    native.call("dftb_trans_charges_noalloc", x["norb"], x["nat"], x["no"], x["nv"], P(x["Co"]), P(x["Cv"]),
                P(x["S"]), P(x["opa"]), P(out[0]), P(out[1]), P(out[2]), native.stream())
    torch.cuda.synchronize()
    return [a.cpu().numpy() for a in out]


def test_noalloc_trans_charges_match_workspace_version_on_two_calls():
    native.load()
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(0)
    first = _inputs(12, 7, dev)
    second = _inputs(16, 8, dev)  # different sizes and values: stale scratch would show
    for x in (first, second):
        ref = _with_workspace(x, dev)
        got = _without_allocation(x, dev)
        for a, b in zip(got, ref):
            assert np.isfinite(a).all()
            assert np.abs(a - b).max() < TOL


def test_noalloc_refuses_requests_beyond_the_static_scratch():
    L = native.load()
    dev = torch.device("cuda", 0)
    limit = L.dftb_trans_charges_noalloc_max_bytes()
    assert limit == 8 << 20
    norb = 2048  # 2048 * (1024 + 1024) doubles = 32 MiB of S.C alone
    assert L.dftb_trans_charges_workspace_size(norb, 1024, 1024) > limit
    out = torch.zeros(4, dtype=torch.float64, device=dev)
    dummy = torch.zeros(4, dtype=torch.float64, device=dev)
    P = native.ptr
    rc = L.dftb_trans_charges_noalloc(norb, 512, 1024, 1024, P(dummy), P(dummy), P(dummy), P(dummy), P(out), P(out),
                                      P(out), native.stream())
    assert rc == native.DFTB_ERR_WORKSPACE if hasattr(native, "DFTB_ERR_WORKSPACE") else rc == -4
    assert b"static array" in L.dftb_last_error()
    # more atoms than the grid's z extent holds: refused before any launch (no orbital blocks, so the
    # scratch itself would fit); the dummy orbitals-per-atom pointer is never read
    assert L.dftb_trans_charges_workspace_size(70000, 0, 0) < limit
    rc = L.dftb_trans_charges_noalloc(70000, 66000, 0, 0, P(dummy), P(dummy), P(dummy), P(dummy), P(out), P(out),
                                      P(out), native.stream())
    assert rc == -1 and b"65535" in L.dftb_last_error()  # DFTB_ERR_BAD_SIZE
    torch.cuda.synchronize()
    assert (out.cpu().numpy() == 0.0).all()
