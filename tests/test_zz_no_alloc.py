"""iccg_dot_dev_noalloc (static device scratch, no allocation) against the
context entry iccg_dot_dev, both through the C ABI.

The file name sorts last so that the entry is also exercised after every
other test of the session has used the device; it passes alone as well.
Test memory comes from torch (the test may allocate; the entry may not).
"""
import ctypes as C
import math

import numpy as np
import pytest

import iccg_b200 as ib

pytestmark = pytest.mark.gpu

MAX_N = 16777216  # ICCG_NOALLOC_MAX_N
# both entries round a double-double sum once; allow a few ulps of |a|.|b|
REL_TOL = 4 * np.finfo(np.float64).eps


def _torch():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    torch.cuda.set_device(0)
    return torch


def _vectors(torch, n, seed):
    g = torch.Generator(device="cpu").manual_seed(seed)
    a = (torch.rand(n, dtype=torch.float64, generator=g) - 0.5).cuda()
    b = (torch.rand(n, dtype=torch.float64, generator=g) * 2.0 - 1.0).cuda()
    return a, b


def _noalloc(torch, n, a, b, out, stream):
    rc = ib.lib().iccg_dot_dev_noalloc(n, C.c_void_p(a.data_ptr() if n else 0),
                                       C.c_void_p(b.data_ptr() if n else 0),
                                       C.c_void_p(out.data_ptr()), C.c_void_p(stream.cuda_stream))
    assert rc == ib.OK, ib.lib().iccg_last_error().decode()
    stream.synchronize()
    return float(out.cpu()[0])


def _with_ctx(ctx, n, a, b):
    res = C.c_double(0.0)
    rc = ib.lib().iccg_dot_dev(ctx.h, n, C.c_void_p(a.data_ptr() if n else 0),
                               C.c_void_p(b.data_ptr() if n else 0), C.byref(res))
    assert rc == ib.OK, ib.lib().iccg_ctx_last_error(ctx.h).decode()
    return res.value


@pytest.mark.parametrize("n", [0, 1, 255, 4096, 4097, 1_000_003, 2_097_152, MAX_N])
def test_noalloc_dot_matches_context_entry(n):
    torch = _torch()
    a, b = _vectors(torch, n, seed=1234 + n)
    out = torch.full((1,), float("nan"), dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    torch.cuda.synchronize()
    ctx = ib.Context(0)
    try:
        want = _with_ctx(ctx, n, a, b)
    finally:
        ctx.close()
    scale = float(torch.dot(a.abs(), b.abs()).item()) if n else 0.0
    got = []
    for _ in range(2):  # two calls in a row: the scratch must be ready again
        out.fill_(float("nan"))
        torch.cuda.synchronize()
        got.append(_noalloc(torch, n, a, b, out, stream))
    for g in got:
        assert math.isfinite(g)
        assert abs(g - want) <= REL_TOL * scale, (n, g, want)
    assert got[0] == got[1]  # fixed chunks: the same sums in the same order
    if n == 0:
        assert got == [0.0, 0.0]


def test_noalloc_dot_known_value():
    torch = _torch()
    n = 3 * 4096 + 17
    a = torch.ones(n, dtype=torch.float64, device="cuda")
    b = torch.arange(n, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()
    for _ in range(2):
        assert _noalloc(torch, n, a, b, out, stream) == n * (n - 1) / 2


def test_noalloc_dot_rejects_oversize_and_bad_arguments():
    torch = _torch()
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    x = torch.zeros(4, dtype=torch.float64, device="cuda")
    L = ib.lib()
    p = C.c_void_p(x.data_ptr())
    rc = L.iccg_dot_dev_noalloc(MAX_N + 1, p, p, C.c_void_p(out.data_ptr()), None)
    assert rc == ib.ERR_ARG
    assert "ICCG_NOALLOC_MAX_N" in L.iccg_last_error().decode()
    assert L.iccg_dot_dev_noalloc(-1, p, p, C.c_void_p(out.data_ptr()), None) == ib.ERR_ARG
    assert L.iccg_dot_dev_noalloc(4, None, p, C.c_void_p(out.data_ptr()), None) == ib.ERR_ARG
    assert L.iccg_dot_dev_noalloc(4, p, p, None, None) == ib.ERR_ARG
    # a rejected call leaves the entry usable
    x.fill_(2.0)
    torch.cuda.synchronize()
    assert L.iccg_dot_dev_noalloc(4, p, p, C.c_void_p(out.data_ptr()), None) == ib.OK
    torch.cuda.synchronize()
    assert float(out.cpu()[0]) == 16.0
