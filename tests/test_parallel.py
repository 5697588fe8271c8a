"""Row-sharded evaluation across ranks (gloo, world size 2, CPU).

The per-rank computation is the oracle's row-range energy here (no GPU); on GPUs
it is dugma_energy_grad_range.  The all-reduced sum must equal the unsharded
result, and every rank must get the same answer."""
import os
import socket

import numpy as np
import torch.multiprocessing as mp

from dugma_b200.parallel import row_ranges


def test_row_ranges_cover_exactly():
    for n in (1, 7, 1000, 1023):
        for w in (1, 2, 3, 8):
            r = row_ranges(n, w)
            assert r[0][0] == 0 and r[-1][1] == n
            assert all(a[1] == b[0] for a, b in zip(r, r[1:]))
            sizes = [b - a for a, b in r]
            assert max(sizes) - min(sizes) <= 1


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as orc
    from dugma_b200 import synth
    from dugma_b200.parallel import energy_grad_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    P = synth.workload0(n=300)
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    R, t = P.R_G, P.t_G

    def compute(i0, i1):
        E, g, _ = st.energy(R, t, 0.05, i0=i0, i1=i1)
        return E, g

    E, g = energy_grad_sharded(st.N, rank, world, compute)
    out[rank] = [E, *g]
    dist.barrier()
    dist.destroy_process_group()


def test_sharded_sum_matches_unsharded():
    from oracle import oracle as orc
    from dugma_b200 import synth
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    P = synth.workload0(n=300)
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    E, g, _ = st.energy(P.R_G, P.t_G, 0.05)
    for r in range(world):
        res = np.asarray(out[r])
        assert abs(res[0] - E) <= 1e-12 * abs(E)
        assert np.allclose(res[1:], g, rtol=1e-12, atol=1e-12 * np.abs(g).max())
    assert np.array_equal(np.asarray(out[0]), np.asarray(out[1]))


def _compi_worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as orc
    from dugma_b200 import synth
    from dugma_b200.parallel import compi_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    P = synth.workload0(n=200)

    def compute(i0, i1, j0, j1):
        # the oracle's coefficients of this rank's source rows against all targets
        # (a partition by source rows; the GPU path also splits the target side by rows)
        st = orc.State(P.X[i0:i1], P.X_C[i0:i1], P.Y, P.Y_C)
        return st.coef(P.R_G, P.t_G, 0.05)

    out[rank] = list(compi_sharded(P.N, P.M, rank, world, compute, 637))
    dist.barrier()
    dist.destroy_process_group()


def test_compi_sharded_sum_matches_unsharded():
    from oracle import oracle as orc
    from dugma_b200 import synth
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_compi_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    P = synth.workload0(n=200)
    A = np.asarray(orc.State(P.X, P.X_C, P.Y, P.Y_C).coef(P.R_G, P.t_G, 0.05))[:637]
    for r in range(world):
        got = np.asarray(out[r])
        assert np.max(np.abs(got - A)) <= 1e-12 * np.max(np.abs(A))
    assert np.array_equal(np.asarray(out[0]), np.asarray(out[1]))


def _sigma_worker(rank, world, port, out):
    import torch.distributed as dist
    from oracle import oracle as orc
    from dugma_b200 import synth
    from dugma_b200.parallel import sigma_sharded
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    P = synth.workload0(n=300)
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    _, d2 = st.nn(P.R_G, P.t_G, 1)
    d2 = d2[:, 0]

    def compute(i0, i1):
        # partial sums of the oracle's nearest squared distances over this rank's rows, with
        # the reference's quantisation of each term (the library's dugma_sigma_range contract)
        q = np.rint((d2[i0:i1] / np.float32(3)).astype(np.float32) * np.float32(1e6)).astype(np.float64)
        return [float(np.sum(d2[i0:i1].astype(np.float64))), float(q.sum())]

    out[rank] = list(sigma_sharded(P.N, 3, rank, world, compute))
    dist.barrier()
    dist.destroy_process_group()


def test_sigma_sharded_matches_unsharded():
    from oracle import oracle as orc
    from dugma_b200 import synth
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.start_processes(_sigma_worker, args=(world, _free_port(), out), nprocs=world, start_method="spawn")
    P = synth.workload0(n=300)
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    sq, se = st.sigma(P.R_G, P.t_G, quantised=True), st.sigma(P.R_G, P.t_G, quantised=False)
    for r in range(world):
        got = out[r]
        assert got[0] == np.float32(sq)
        assert abs(got[1] - se) <= 1e-14 * se
