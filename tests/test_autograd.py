"""torch.autograd harness of the fused adjoint (GPU): backward against central
finite differences of the same function, and against the FP64 oracle."""
import numpy as np
import pytest
import torch

from oracle import oracle as orc
from dugma_b200 import api, synth
from dugma_b200.autograd import PoseEnergy, SourceEnergy
from dugma_b200.pose import expmap

pytestmark = pytest.mark.gpu


def test_pose_energy_backward_matches_fd():
    P = synth.workload0()
    _, h = api.init(P.X, P.X_C, P.Y, P.Y_C)
    try:
        R0 = P.R_G @ expmap([0.1, 0.0, -0.1])
        sig = 0.05
        omega = torch.tensor([0.03, -0.02, 0.05], dtype=torch.float64, requires_grad=True)
        t = torch.tensor(P.t_G + 0.01, dtype=torch.float64, requires_grad=True)
        E = PoseEnergy.apply(omega, t, h, R0, sig)
        E.backward()
        ga = torch.cat([omega.grad, t.grad]).numpy()
        eps = 1e-4
        fd = []
        base = torch.cat([omega.detach(), t.detach()])
        for k in range(6):
            v = []
            for s in (1, -1):
                p = base.clone()
                p[k] += s * eps
                v.append(float(PoseEnergy.apply(p[:3], p[3:], h, R0, sig)))
            fd.append((v[0] - v[1]) / (2 * eps))
        fd = np.array(fd)
        assert np.linalg.norm(ga - fd) <= 1e-4 * np.linalg.norm(fd), (ga, fd)
        # and the FP64 oracle at the same pose
        st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
        R = expmap(omega.detach().numpy()) @ R0
        Eo, go, _ = st.energy(R, t.detach().numpy(), sig)
        assert abs(float(E) - Eo) <= 1e-6 * Eo
    finally:
        api.fr_m(h)


def test_source_energy_backward_matches_oracle():
    P = synth.workload0(n=400)
    X = torch.tensor(P.X, dtype=torch.float64, requires_grad=True)
    E = SourceEnergy.apply(X, P.X_C, P.Y, P.Y_C, P.R_G, P.t_G, 0.05)
    E.backward()
    st = orc.State(P.X, P.X_C, P.Y, P.Y_C)
    Eo, _, dxo = st.energy(P.R_G, P.t_G, 0.05, with_dx=True)
    assert abs(float(E) - Eo) <= 1e-6 * Eo
    assert np.linalg.norm(X.grad.numpy() - dxo) <= 1e-4 * np.linalg.norm(dxo)
