"""End-to-end registration of the reference's 30 real Kinect scenes (tests/golden/kinect_scenes.npz,
made by tests/golden/make_kinect.py from dataset_all/Kinect_Application and the authors' recorded
results Our_result_in_Kinect_Application) with the settings of main_kinect_real_application.m:14-34
(identity start, 300 iterations, tolerances 1e-4 / 1e-8 / 1e-9) and its error measures.

Mode 0 is the reference's loop (DUGMA.m: update_sig, compi, the surrogate minimised on SO(3) in place
of fmincon, the t <- dt + t update): it must reproduce the authors' recorded pose of every scene,
scene 26 included (the scene where the authors' run itself failed), to 0.05 degrees and 2e-3 in
translation, and so their error statistics against the ground truth.  Mode 1 (this library's direct
quasi-Newton on the fused adjoint, not the reference's method) is reported and held to a median.
"""
import os

import pytest

from dugma_b200 import evaluate

pytestmark = pytest.mark.gpu
FIXTURE = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "kinect_scenes.npz")


def _run(mode):
    rows = [evaluate.register(P, mode, 300, rec) for P, rec in evaluate.scenes_from_npz(FIXTURE)]
    for r in rows:
        print(f"mode {mode} {r['scene']:8s} N={r['N']:5d} M={r['M']:5d} error_R={r['error_R']:.5f} "
              f"error_t={r['error_t']:.5f} {r['iterations']:3d} it {r['seconds']:.3f} s (recorded "
              f"{r['recorded_seconds']:.1f} s); vs recorded {r['vs_recorded_deg']:.2e} deg "
              f"{r['vs_recorded_t']:.2e}")
    return rows


def test_kinect_reference_loop_reproduces_recorded_poses():
    rows = _run(0)
    assert len(rows) == 30
    for r in rows:
        assert r["vs_recorded_deg"] <= 0.05, r
        assert r["vs_recorded_t"] <= 2e-3, r
    s = evaluate.summarise(rows, 0)
    assert abs(s["error_R"]["median"] - s["recorded_error_R"]["median"]) <= 1e-4
    assert abs(s["error_t"]["median"] - s["recorded_error_t"]["median"]) <= 1e-4
    print("mode 0 summary:", s)


def test_kinect_direct_adjoint_mode():
    rows = _run(1)
    s = evaluate.summarise(rows, 1)
    print("mode 1 summary:", s)
    assert s["vs_recorded_deg"]["median"] <= 1.0
    assert sum(r["vs_recorded_deg"] <= 2.0 for r in rows) >= 24
