"""The allocation-free HE-VI substep entry point.

cress_hevi_substep_noalloc is for callers that cannot call cudaMalloc from
inside their time loop (a host model whose device arrays sit in a pool it
sized at start-up, or a framework whose caching allocator owns the device).
Here torch plays that caller: it owns every device buffer, and the entry
point is called through the C-ABI twice in a row (substep 1, then substep 2
from substep 1's output) into output buffers filled with NaN, so a point
the kernel fails to write shows up.  Each result must match the CPU oracle's
s_smalldrv loop (nsstp = 1 and 2) within the tolerance of the other
small-step tests, for divopt 0, 1, 2 and sthopt 0, 1; one case is also
checked against the context API (cress_smalldrv).  Device memory must not
change across repeated calls.  This file is collected last so a failure
here comes after every other test.
"""
import ctypes

import numpy as np
import pytest

import helpers as H

pytestmark = pytest.mark.gpu

RTOL = 2e-5  # per substep, relative to the field's max magnitude
STAG = {"u": "u", "v": "v", "w": "s", "pp": "s"}


def _entry(cress):
    L = cress.lib()
    fn = L.cress_hevi_substep_noalloc
    P = ctypes.c_void_p
    fn.argtypes = [ctypes.POINTER(cress.Cfg), ctypes.c_float, ctypes.POINTER(cress._FP)] + [P] * 12 + [P]
    fn.restype = ctypes.c_int
    return L, fn


def _cfg(cress, ni, nj, nk, dx, dz, sthopt, divopt):
    c = cress.Cfg()
    c.ni, c.nj, c.nk = ni, nj, nk
    c.dx, c.dy, c.dz = dx, dx, dz
    c.sthopt, c.impopt, c.divopt, c.buyopt, c.gwmopt = sthopt, 1, divopt, 1, 0
    c.weicoe = 0.6
    c.wbc = c.ebc = c.sbc = c.nbc = -1
    c.bbc = c.tbc = 2
    return c


def _check(ni, nj, nk, outs, refs, nsub, what):
    for name, t, r in zip(("u", "v", "w", "pp"), outs, refs):
        g = t[:, :, :ni + 2].cpu().numpy()
        m = H.interior_mask(ni, nj, nk, STAG[name])
        assert np.isfinite(g[m]).all(), (what, nsub, name, "unwritten or non-finite points")
        scale = float(np.abs(r[m]).max()) + 1e-30
        err = float(np.abs(g[m] - r[m]).max())
        assert err <= RTOL * (nsub + 1) * scale, (what, nsub, name, err, scale)


@pytest.mark.parametrize("divopt,sthopt", [(2, 1), (1, 1), (0, 1), (2, 0)])
def test_noalloc_two_calls_match_oracle(cress, oracle_lib, divopt, sthopt):
    import torch
    from cress_b200 import cases

    nx, ny, nz = 70, 45, 30
    dx, dz, dts = 1000.0, 250.0, 0.5
    (ni, nj, nk), base, st, frc = cases.acoustic_case(nx, ny, nz, dx, dz, seed=21 + divopt, sthopt=sthopt)
    ocfg = dict(ni=ni, nj=nj, nk=nk, dx=dx, dy=dx, dz=dz, sthopt=sthopt, divopt=divopt, buyopt=1,
                weicoe=0.6)
    ref1 = oracle_lib.small_steps(ocfg, base, frc, [a.copy() for a in st], 1, dts, prec=32, fp64_solve=1)
    ref2 = oracle_lib.small_steps(ocfg, base, frc, [a.copy() for a in st], 2, dts, prec=32, fp64_solve=1)

    # caller-owned device buffers in the padded layout; the outputs start as NaN
    px = (ni + 2 + 31) // 32 * 32
    dev = torch.device("cuda", 0)

    def to_dev(a):
        t = torch.zeros((nk, nj + 2, px), dtype=torch.float32, device=dev)
        t[:, :, :ni + 2] = torch.from_numpy(np.ascontiguousarray(a))
        return t

    old = [to_dev(a) for a in st]
    frc_d = [to_dev(a) for a in frc]
    new1 = [torch.full((nk, nj + 2, px), float("nan"), dtype=torch.float32, device=dev) for _ in st]
    new2 = [torch.full((nk, nj + 2, px), float("nan"), dtype=torch.float32, device=dev) for _ in st]
    spare = [torch.empty_like(t) for t in new1]

    L, fn = _entry(cress)
    c = _cfg(cress, ni, nj, nk, dx, dz, sthopt, divopt)
    barrs = [np.ascontiguousarray(base[n], dtype=np.float32) for n in cress.BASE_NAMES]
    bptr = (cress._FP * len(barrs))(*[cress.fptr(a) for a in barrs])
    stream = torch.cuda.current_stream(dev).cuda_stream
    P = ctypes.c_void_p

    def call(o, n):
        rc = fn(ctypes.byref(c), dts, bptr, *[P(t.data_ptr()) for t in o], *[P(t.data_ptr()) for t in frc_d],
                *[P(t.data_ptr()) for t in n], P(stream))
        assert rc == 0, L.cress_last_error().decode()

    call(old, new1)   # the first call on the device also finds the scratch's address
    call(new1, new2)  # a second call in a row shares the same scratch
    torch.cuda.synchronize()
    _check(ni, nj, nk, new1, ref1, 1, "oracle")
    _check(ni, nj, nk, new2, ref2, 2, "oracle")

    # repeated calls change no device memory (every buffer exists already)
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info(dev)[0]
    for _ in range(3):
        call(old, spare)
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info(dev)[0] == free0


def test_noalloc_matches_context_api(cress):
    import torch
    from cress_b200 import cases

    nx, ny, nz = 70, 45, 30
    dx, dz, dts = 1000.0, 250.0, 0.5
    (ni, nj, nk), base, st, frc = cases.acoustic_case(nx, ny, nz, dx, dz, seed=21, sthopt=1)
    s = cress.Solver(ni, nj, nk, dx, dx, dz, sthopt=1)
    s.set_base3d(base)
    ref1 = s.smalldrv(1, dts, *st, *frc)
    ref2 = s.smalldrv(2, dts, *st, *frc)
    s.close()

    px = (ni + 2 + 31) // 32 * 32
    dev = torch.device("cuda", 0)

    def to_dev(a):
        t = torch.zeros((nk, nj + 2, px), dtype=torch.float32, device=dev)
        t[:, :, :ni + 2] = torch.from_numpy(np.ascontiguousarray(a))
        return t

    old = [to_dev(a) for a in st]
    frc_d = [to_dev(a) for a in frc]
    new1 = [torch.full((nk, nj + 2, px), float("nan"), dtype=torch.float32, device=dev) for _ in st]
    new2 = [torch.full((nk, nj + 2, px), float("nan"), dtype=torch.float32, device=dev) for _ in st]
    L, fn = _entry(cress)
    c = _cfg(cress, ni, nj, nk, dx, dz, 1, 2)
    barrs = [np.ascontiguousarray(base[n], dtype=np.float32) for n in cress.BASE_NAMES]
    bptr = (cress._FP * len(barrs))(*[cress.fptr(a) for a in barrs])
    stream = torch.cuda.current_stream(dev).cuda_stream
    P = ctypes.c_void_p
    for o, n in ((old, new1), (new1, new2)):
        rc = fn(ctypes.byref(c), dts, bptr, *[P(t.data_ptr()) for t in o], *[P(t.data_ptr()) for t in frc_d],
                *[P(t.data_ptr()) for t in n], P(stream))
        assert rc == 0, L.cress_last_error().decode()
    torch.cuda.synchronize()
    _check(ni, nj, nk, new1, ref1, 1, "context API")
    _check(ni, nj, nk, new2, ref2, 2, "context API")


def test_noalloc_rejects_too_many_levels(cress):
    import torch
    L, fn = _entry(cress)
    P = ctypes.c_void_p
    c = _cfg(cress, 20, 20, 300, 1000.0, 100.0, 0, 2)
    dummy = torch.zeros(64, device="cuda")
    host = np.zeros(8, np.float32)
    bptr = (cress._FP * len(cress.BASE_NAMES))(*[cress.fptr(host)] * len(cress.BASE_NAMES))
    ptrs = [P(dummy.data_ptr())] * 12
    rc = fn(ctypes.byref(c), 0.5, bptr, *ptrs, P(0))
    assert rc == 1  # CRESS_E_ARG
    assert b"256" in L.cress_last_error()
