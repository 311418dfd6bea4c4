"""The allocation-free dry-mass entry point (GPU).

wfe_dry_mass_noalloc serves callers that cannot call cudaMalloc (code running
inside another framework's stream capture, or a process whose device memory
belongs to a fixed-budget pool allocator).  Here the "caller" owns its device
buffers through torch's allocator, hands them to the entry point through the C
ABI, and the result of two calls in a row must equal wfe_dry_mass, the
library's allocating entry point, within the 1e-12 relative tolerance the
dry-mass test uses.  This file is collected last and works in a fresh process
as well as after the other tests.
"""

import ctypes as C

import numpy as np
import pytest

import wfe_b200 as W
from helpers import CASES

pytestmark = pytest.mark.gpu


def _ptr(t):
    return C.c_void_p(t.data_ptr())


def test_dry_mass_noalloc_matches_allocating_entry_point():
    import torch

    c = W.Case(CASES / "wk82_small.ini", precision="f64", device=0)
    for s in range(3):
        c.step(c.dt, s * c.dt)
    ref = c.dry_mass()

    dev = torch.device("cuda", 0)
    state = {k: torch.from_numpy(c.field(k).ravel().copy()).to(dev)
             for k in ("pip", "thp", "qv", "qc", "qr")}
    pib = torch.from_numpy(c.base("pib")).to(dev)
    thb = torch.from_numpy(c.base("thb")).to(dev)
    jac = torch.from_numpy(c.metric("jac")).to(dev)
    dzc = torch.from_numpy(c.metric("dzeta_c")).to(dev)
    out = torch.full((2,), -1.0, dtype=torch.float64, device=dev)
    torch.cuda.synchronize()

    lib = W.load_library()
    args = [_ptr(pib), _ptr(thb), _ptr(state["pip"]), _ptr(state["thp"]), _ptr(state["qv"]),
            _ptr(state["qc"]), _ptr(state["qr"]), _ptr(jac), _ptr(dzc)]
    for call in range(2):
        slot = C.c_void_p(out.data_ptr() + 8 * call)
        rc = lib.wfe_dry_mass_noalloc(c.nx, c.ny, c.nz, c.dx, c.dy, *args, slot, None)
        assert rc == 0, lib.wfe_last_error(None)
    torch.cuda.synchronize()
    got = out.cpu().numpy()
    for call in range(2):
        assert abs(got[call] - ref) <= 1e-12 * abs(ref), (call, got[call], ref)

    # sizes beyond the static scratch are rejected with a clear error
    rc = lib.wfe_dry_mass_noalloc(c.nx, c.ny, W_MAX + 1, c.dx, c.dy, *args,
                                  C.c_void_p(out.data_ptr()), None)
    assert rc == 1
    assert b"exceeds the static scratch" in lib.wfe_last_error(None)
    c.close()


W_MAX = 1024  # WFE_NOALLOC_MAX_LEVELS in include/wfe_b200.h
