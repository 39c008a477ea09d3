"""sr_gravity_solve_static: the gravity solve for callers that cannot allocate device memory (a host that owns every
device buffer and forbids its plug-ins cudaMalloc, or a loop that cannot take cudaMalloc's device-wide
synchronisation). Its scratch lives in the library's static device arrays; the caller passes the density and the
output buffers. Checked here through the C ABI against the allocating path (a context's P2, sr_gravity_field) on two
calls in a row, within the gravity tests' tolerance (rel L1 <= 1e-5), and its refusal of a world past the static
scratch. This file is collected last so that a run stopping at its first failure has run every other test."""
import ctypes as C

import numpy as np
import pytest

from sandbox_reactions_b200 import scenes
from sandbox_reactions_b200.abi import Config
from sandbox_reactions_b200.engine import Step, load_library

pytestmark = pytest.mark.gpu


def rel_l1(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return np.abs(a - b).sum() / np.abs(b).sum()


def test_the_static_solve_matches_the_allocating_path_on_two_calls():
    import torch

    lib = load_library()
    cfg, P = scenes.disk(256)
    cfg = cfg.replace(width=192, height=128, hydro=False)
    P = np.ascontiguousarray(P[:, 64:192, 32:224])
    with Step(cfg) as s:
        s.upload(P)
        phi0, gx0, gy0 = s.gravity_field()
    c = cfg.to_c()
    sigma = torch.from_numpy(np.ascontiguousarray(P[0])).cuda()
    outs = [torch.full((cfg.height, cfg.width), float("nan"), device="cuda") for _ in range(3)]
    stream = torch.cuda.current_stream()
    for _ in range(2):
        st = lib.sr_gravity_solve_static(C.byref(c), sigma.data_ptr(), outs[0].data_ptr(), outs[1].data_ptr(),
                                         outs[2].data_ptr(), C.c_void_p(stream.cuda_stream))
        assert st == 0, lib.sr_last_error(None).decode()
        torch.cuda.synchronize()
        phi, gx, gy = (o.cpu().numpy() for o in outs)
        assert rel_l1(phi, phi0) <= 1e-5
        assert rel_l1(gx, gx0) <= 1e-5 and rel_l1(gy, gy0) <= 1e-5
        for o in outs:
            o.fill_(float("nan"))


def test_the_static_solve_rebuilds_its_tables_when_the_world_or_kernel_changes():
    # 192x128 self-cell, 64x64 softened, 192x128 self-cell again on one device: every change of padded size and
    # kernel rebuilds the spectrum in the static arrays; each call is held to a fresh context's P2.
    import torch

    lib = load_library()
    base, P = scenes.disk(256)
    cases = [(192, 128, "self_cell"), (64, 64, "softened"), (192, 128, "self_cell")]
    stream = torch.cuda.current_stream()
    for w, h, kernel in cases:
        cfg = base.replace(width=w, height=h, hydro=False, kernel=kernel)
        Q = np.ascontiguousarray(P[:, 128 - h // 2:128 + h // 2, 128 - w // 2:128 + w // 2])
        with Step(cfg) as s:
            s.upload(Q)
            phi0, gx0, gy0 = s.gravity_field()
        c = cfg.to_c()
        sigma = torch.from_numpy(np.ascontiguousarray(Q[0])).cuda()
        outs = [torch.full((h, w), float("nan"), device="cuda") for _ in range(3)]
        st = lib.sr_gravity_solve_static(C.byref(c), sigma.data_ptr(), outs[0].data_ptr(), outs[1].data_ptr(),
                                         outs[2].data_ptr(), C.c_void_p(stream.cuda_stream))
        assert st == 0, lib.sr_last_error(None).decode()
        torch.cuda.synchronize()
        phi, gx, gy = (o.cpu().numpy() for o in outs)
        assert rel_l1(phi, phi0) <= 1e-5, (w, h, kernel, rel_l1(phi, phi0))
        assert rel_l1(gx, gx0) <= 1e-5 and rel_l1(gy, gy0) <= 1e-5, (w, h, kernel)


def test_the_static_solve_refuses_a_world_past_its_scratch():
    import torch

    lib = load_library()
    c = Config(width=512, height=64, gravity=True, hydro=False).to_c()
    buf = torch.zeros((64, 512), device="cuda")
    st = lib.sr_gravity_solve_static(C.byref(c), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(), buf.data_ptr(),
                                     None)
    assert st == 1
    assert b"256x256" in lib.sr_last_error(None)
