"""The library's sharded path across processes: two ranks (spawned processes, gloo for the
host-side all-reduce), each with its own context on the GPU, evaluate their source-row (and, for
compi, target-row) ranges through dugma_energy_grad_range, dugma_compi_range and
dugma_sigma_range; the all-reduced sums must equal the unsharded library results (energy and
pose gradient to 1e-12 relative, sigma bit for bit; the coefficients to 1e-12 of the same row
ranges summed in one process and to 1e-6 of max |A| of the one-pass compi over all rows, which
adds the same pair terms in another FP32 order).  The ranks' kernels are
independent of each other; only the few partial sums travel through the collective."""
import os
import socket

import numpy as np
import pytest
import torch.multiprocessing as mp

pytestmark = pytest.mark.gpu


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import datetime

    import torch.distributed as dist
    from dugma_b200 import api, synth
    from dugma_b200.parallel import compi_sharded, energy_grad_sharded, sigma_sharded
    from dugma_b200.pose import expmap
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=60))
    P = synth.workload0()
    R, t = P.R_G @ expmap([0.04, -0.02, 0.03]), P.t_G + 0.005
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    try:
        sig_q, sig_e = sigma_sharded(P.N, 3, rank, world, lambda i0, i1: api.sigma_range(h, R, t, i0, i1))
        E, g = energy_grad_sharded(P.N, rank, world, lambda i0, i1: api.energy_grad_range(h, R, t, sig_q, i0, i1))
        A = compi_sharded(P.N, P.M, rank, world,
                          lambda i0, i1, j0, j1: api.compi_range(h, R, t, sig_q, i0, i1, j0, j1), 637)
        res = {"sig_q": sig_q, "sig_e": sig_e, "E": E, "g": list(g), "A": list(A)}
        if rank == 0:
            # the unsharded library results on this rank's own context
            sig_ref = api.update_sig(h, R, t)
            E1, g1, _ = api.energy_grad(h, R, t, sig_ref)
            from dugma_b200.parallel import row_ranges
            ri, rj = row_ranges(P.N, world), row_ranges(P.M, world)
            A_parts = sum(api.compi_range(h, R, t, sig_ref, *ri[r], *rj[r]) for r in range(world))
            res.update({"ref_sig": sig_ref, "ref_E": E1, "ref_g": list(g1),
                        "ref_A": list(api.compi(h, R, t, sig=sig_ref)), "ref_A_parts": list(A_parts),
                        "ref_sig_e": api.sigma(h, R, t)})
        out[rank] = res
    finally:
        api.fr_m(h)
        dist.barrier()
        dist.destroy_process_group()


def test_two_ranks_sharded_library_matches_unsharded():
    world = 2
    ctx = mp.get_context("spawn")
    mgr = ctx.Manager()
    out = mgr.dict()
    mp.start_processes(_rank, args=(world, _free_port(), out), nprocs=world, start_method="spawn", join=True)
    r0, r1 = out[0], out[1]
    for r in (r0, r1):
        assert r["sig_q"] == r0["ref_sig"]                       # bit for bit
        assert abs(r["sig_e"] - r0["ref_sig_e"]) <= 1e-12 * r0["ref_sig_e"]
        assert abs(r["E"] - r0["ref_E"]) <= 1e-12 * abs(r0["ref_E"])
        g, gr = np.array(r["g"]), np.array(r0["ref_g"])
        assert np.linalg.norm(g - gr) <= 1e-12 * np.linalg.norm(gr)
        # the same row ranges summed in one process: the collective adds nothing but FP64 rounding;
        # the one-pass compi over all rows sums the same pairs in another FP32 order
        A, Ap, Ar = np.array(r["A"]), np.array(r0["ref_A_parts"]), np.array(r0["ref_A"])
        assert np.abs(A - Ap).max() <= 1e-12 * np.abs(Ap).max()
        assert np.abs(A - Ar).max() <= 1e-6 * np.abs(Ar).max()
    assert r0["E"] == r1["E"] and r0["g"] == r1["g"] and r0["A"] == r1["A"]
