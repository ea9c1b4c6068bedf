"""The allocation-free field entry point (fs_field_eval_noalloc).

It serves callers that cannot allocate device memory when they need the field
(a pool or arena that owns the device, hosts that allocate only at start-up,
threads where cudaMalloc's device-wide synchronisation is not allowed): its
scratch lives in one static device array.  Checked through the C ABI against
the regular FP32-compensated entry point, on two calls in a row (the second
call finds the first call's leftovers in the shared array).  This file sorts
last so a run that stops at the first failure has run every other test."""
import ctypes

import numpy as np
import pytest

import multi_species_b200 as M

pytestmark = pytest.mark.gpu
TOL32 = 1e-6  # relative L2 bound on E used for the FP32-compensated kernel


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / np.linalg.norm(b))


def test_noalloc_matches_regular_entry_point_twice():
    import torch
    lib = M.lib()
    rng = np.random.default_rng(11)
    L, eps = 10 * np.pi, 0.02
    regular = M.E_MQ_DirectSum_B200(L, eps, "fp32c")
    for n in (20000, 32768):  # two calls in a row, different sizes
        x = rng.uniform(-L, 2 * L, n)
        q = -np.abs(rng.normal(size=n)) * (L / n)
        want = regular.evaluate(x, x, q)
        dx = torch.tensor(x, dtype=torch.float64, device="cuda")
        dq = torch.tensor(q, dtype=torch.float64, device="cuda")
        de = torch.full((n,), float("nan"), dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = lib.fs_field_eval_noalloc(L, eps, ctypes.c_void_p(de.data_ptr()), ctypes.c_void_p(dx.data_ptr()),
                                       ctypes.c_void_p(dq.data_ptr()), n, None)
        assert rc == 0, lib.fs_last_error().decode()
        got = de.cpu().numpy()
        assert rel_l2(got, want) < TOL32


def test_noalloc_rejects_sizes_over_the_limit():
    import torch
    lib = M.lib()
    n = 32769
    d = torch.zeros(n, dtype=torch.float64, device="cuda")
    p = ctypes.c_void_p(d.data_ptr())
    rc = lib.fs_field_eval_noalloc(1.0, 0.1, p, p, p, n, None)
    assert rc == 1
    assert "32768" in lib.fs_last_error().decode()
