"""The allocation-free density entry point, for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc: a host framework that owns the device allocator, or a
run that must not allocate once it is planned.  nb_density_noalloc serves them with a fixed
device scratch array instead.  This test calls it through the C ABI and checks it against the
ordinary nb_density entry point on the reference's density fixture, twice in a row (the shared
scratch keeps the previous call's contents), at the tolerance of the other density tests.
It lives in its own file, collected last, so a run stopping at a failure here has already run
every other test; it passes alone in a fresh process as well as after them.
"""

import ctypes

import numpy as np
import pytest

from tests.conftest import check, golden

pytestmark = pytest.mark.gpu


def test_density_noalloc_matches_density():
    import torch

    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    from blackhole_nebula_simulator_b200 import _lib
    from blackhole_nebula_simulator_b200.device import ctx, dev_f64, dev_i64, ptr, stream

    g = golden("density.npz")
    n = len(g["pos"])
    pos, mass = dev_f64(g["pos"]), dev_f64(g["mass"])
    h0, hs = dev_f64(g["h_first"]), dev_f64(g["h_search"])
    off, idx = dev_i64(g["offset"]), dev_i64(g["index"])
    L = _lib.lib()

    def outputs():
        d = pos.device
        return [torch.empty(n, dtype=torch.float64, device=d) for _ in range(3)] + [
            torch.empty(n, dtype=torch.int64, device=d) for _ in range(2)]

    ref = outputs()
    c = ctx()
    _lib.check(c, L.nb_density(c, n, ptr(pos), ptr(mass), ptr(h0), ptr(hs), ptr(off), ptr(idx), n,
                               None, 1, 1.6, 1e-12, 0.5, *[ptr(t) for t in ref], stream()))
    for call in range(2):
        out = outputs()
        for t in out:
            t.fill_(-1)
        st = L.nb_density_noalloc(n, ptr(pos), ptr(mass), ptr(h0), ptr(hs), ptr(off), ptr(idx), n,
                                  None, 1, 1.6, 1e-12, 0.5, *[ptr(t) for t in out], stream())
        assert st == 0, L.nb_noalloc_last_error()
        torch.cuda.synchronize()
        for name, a, b in zip(("h", "rho", "omega"), ref[:3], out[:3]):
            check(f"call {call}: {name}", a.cpu().numpy(), b.cpu().numpy(), rtol=1e-12)
        check(f"call {call}: iterations", ref[3].cpu().numpy(), out[3].cpu().numpy())
        check(f"call {call}: flags", ref[4].cpu().numpy(), out[4].cpu().numpy())
    check("noalloc vs reference fixture: h", g["h"], out[0].cpu().numpy(), rtol=1e-12)
    # sizes beyond the fixed scratch are refused with a clear error
    too_many = L.nb_density_noalloc(300000, ptr(pos), ptr(mass), ptr(h0), ptr(hs), ptr(off),
                                    ptr(idx), 1, None, 1, 1.6, 1e-12, 0.5,
                                    *[ptr(t) for t in out], stream())  # fmt: skip
    assert too_many == 26 and b"beyond the fixed scratch" in L.nb_noalloc_last_error()
