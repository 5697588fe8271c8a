"""The allocation-free entry point dugma_energy_grad_noalloc against dugma_energy_grad.

Some callers cannot allocate device memory while they evaluate (latency-bounded loops
that must never enter an allocator, hosts that own all device memory).  For them the
library offers one entry point whose working memory is a fixed file-scope device array.
This test calls it through the C ABI with a context's device arrays as inputs and device
tensors for the pose and the result, twice in a row (the second call reuses the array the
first one left behind), and compares each result with the allocating entry point's and with
the FP64 oracle's at the tolerances of the other parity tests (energy 1e-6, pose gradient
1e-5, relative); the second call must leave the device's free memory unchanged.  The size
limit is checked on both sides of it.  It lives in its own file, named to be collected last.
"""
import ctypes

import numpy as np
import pytest

from dugma_b200 import _lib, api, synth
from dugma_b200.pose import expmap, rot2d
from oracle import oracle as orc

pytestmark = pytest.mark.gpu


def _problem(D):
    if D == 3:
        P = synth.workload0()
        return P.X, P.X_C, P.Y, P.Y_C, P.R_G @ expmap([0.05, -0.1, 0.08]), P.t_G + 0.01
    rng = np.random.default_rng(4)
    n = 900
    th = rng.uniform(0, 2 * np.pi, n)
    X = np.stack([np.cos(th), np.sin(th) * (1 + 0.2 * np.cos(3 * th))], 1)
    Y = X[rng.permutation(n)[:700]] @ rot2d(0.3).T + 0.05 + 0.01 * rng.standard_normal((700, 2))
    XC = np.einsum("n,ab->nab", rng.uniform(1e-3, 3e-3, n), np.eye(2))
    YC = np.einsum("n,ab->nab", rng.uniform(1e-3, 3e-3, 700), np.eye(2))
    return X, XC, Y, YC, rot2d(-0.25), np.array([-0.03, 0.02])


@pytest.mark.parametrize("D", [3, 2])
def test_noalloc_matches_allocating_entry_point(D):
    import torch

    X, XC, Y, YC, R, t = _problem(D)
    _, h = api.init(X, XC, Y, YC)
    L = _lib.load()
    try:
        sig = api.update_sig(h, R, t)
        E_ref, g_ref, _ = api.energy_grad(h, R, t, sig)
        E_o, g_o, _ = orc.State(X, XC, Y, YC).energy(R, t, sig)
        pose = torch.zeros(16, dtype=torch.float64, device="cuda")
        pose[: D * D] = torch.tensor(np.asarray(R).T.reshape(-1))
        pose[9:9 + D] = torch.tensor(t)
        pose[12] = sig
        ng = 6 if D == 3 else 3
        stream = torch.cuda.Stream()
        for call in range(2):
            out = torch.full((8,), float("nan"), dtype=torch.float64, device="cuda")
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = L.dugma_energy_grad_noalloc(*h.ptrs, h.N, h.M, h.D, pose.data_ptr(), out.data_ptr(),
                                             ctypes.c_void_p(stream.cuda_stream))
            assert rc == _lib.OK, L.dugma_last_error()
            stream.synchronize()
            if call == 1:
                # the first call may load the library's kernels (and with them the array); after it
                # nothing may take device memory
                assert torch.cuda.mem_get_info()[0] >= free0
            res = out.cpu().numpy()
            E, g = res[0], res[1:1 + ng]
            assert abs(E - E_ref) <= 1e-6 * abs(E_ref), (call, E, E_ref)
            assert np.linalg.norm(g - g_ref) <= 1e-5 * np.linalg.norm(g_ref), (call, g, g_ref)
            assert abs(E - E_o) <= 1e-6 * abs(E_o), (call, E, E_o)
            assert np.linalg.norm(g - g_o) <= 1e-5 * np.linalg.norm(g_o), (call, g, g_o)
    finally:
        api.fr_m(h)


def test_noalloc_rejects_sizes_beyond_its_scratch():
    P = synth.workload0(n=200)
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    L = _lib.load()
    try:
        import torch
        pose = torch.zeros(16, dtype=torch.float64, device="cuda")
        out = torch.zeros(8, dtype=torch.float64, device="cuda")
        for n, m in ((20000, h.M), (h.N, 16385), (16385, 16385)):
            rc = L.dugma_energy_grad_noalloc(*h.ptrs, n, m, 3, pose.data_ptr(), out.data_ptr(), None)
            assert rc == _lib.ERR_ARG, (n, m)
            assert b"16384" in L.dugma_last_error()
    finally:
        api.fr_m(h)


def test_noalloc_accepts_the_largest_size():
    """N = M = 16384, where the carved scratch (records, log weights, worst-case partial sums) is
    closest to the array's size: accepted, and equal to the allocating entry point's result."""
    import torch

    P = synth.workload0(n=16384)
    R, t = P.R_G @ expmap([0.02, 0.03, -0.01]), P.t_G
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    L = _lib.load()
    try:
        assert (h.N, h.M) == (16384, 16384)
        sig = api.update_sig(h, R, t)
        E_ref, g_ref, _ = api.energy_grad(h, R, t, sig)
        pose = torch.zeros(16, dtype=torch.float64, device="cuda")
        pose[:9] = torch.tensor(np.asarray(R).T.reshape(-1))
        pose[9:12] = torch.tensor(t)
        pose[12] = sig
        out = torch.zeros(8, dtype=torch.float64, device="cuda")
        torch.cuda.synchronize()
        rc = L.dugma_energy_grad_noalloc(*h.ptrs, h.N, h.M, 3, pose.data_ptr(), out.data_ptr(), None)
        assert rc == _lib.OK, L.dugma_last_error()
        torch.cuda.synchronize()
        res = out.cpu().numpy()
        assert abs(res[0] - E_ref) <= 1e-6 * abs(E_ref), (res[0], E_ref)
        assert np.linalg.norm(res[1:7] - g_ref) <= 1e-5 * np.linalg.norm(g_ref)
    finally:
        api.fr_m(h)
