"""Seeded synthetic point clouds for the registration workloads.

Every generator returns float64 arrays in the memory layout the reference's
MATLAB/MEX entry points take: X is D x N column-major, i.e. a C array of
shape (N, D) with each point's coordinates contiguous; X_C is D x (D*N)
column-major, i.e. a C array of shape (N, D, D) holding one D x D block per
point (DUGMA.m:19 arguments; dataset "Read Me":7-8 describes the same
per-point block layout).  The reference moves Y onto X: the ground-truth pose
(R_G, t_G) satisfies R_G @ y + t_G ~ x (main_simulation.m:63-64 measures
errors against it).

The shapes, sizes and noise models are those of the five named workloads
(unit-sphere-with-bumps at 1000 and 6000 points, a spherical-harmonic surface
at 65536 points, a batch of 256 uneven problems, and two depth-camera views at
300000 points).  No public dataset is involved; all inputs are drawn from
numpy's PCG64 generator with seed = 1000 * workload + trial.
"""
from __future__ import annotations

import dataclasses
import math

import numpy as np


@dataclasses.dataclass
class Problem:
    X: np.ndarray          # (N, 3) float64, fixed cloud
    Y: np.ndarray          # (M, 3) float64, moving cloud
    X_C: np.ndarray        # (N, 3, 3) float64 per-point covariance
    Y_C: np.ndarray        # (M, 3, 3) float64 per-point covariance
    R_G: np.ndarray        # (3, 3) ground-truth rotation, R_G @ y + t_G ~ x
    t_G: np.ndarray        # (3,)
    name: str = ""

    @property
    def N(self) -> int:
        return self.X.shape[0]

    @property
    def M(self) -> int:
        return self.Y.shape[0]


def rng_for(workload: int, trial: int = 0) -> np.random.Generator:
    return np.random.Generator(np.random.PCG64(1000 * workload + trial))


def rotation_axis_angle(axis: np.ndarray, angle: float) -> np.ndarray:
    axis = np.asarray(axis, dtype=np.float64)
    axis = axis / np.linalg.norm(axis)
    K = np.array([[0.0, -axis[2], axis[1]],
                  [axis[2], 0.0, -axis[0]],
                  [-axis[1], axis[0], 0.0]])
    return np.eye(3) + math.sin(angle) * K + (1.0 - math.cos(angle)) * (K @ K)


def random_unit_vectors(rng: np.random.Generator, n: int) -> np.ndarray:
    v = rng.standard_normal((n, 3))
    return v / np.linalg.norm(v, axis=1, keepdims=True)


def random_rotation(rng: np.random.Generator, max_angle_deg: float) -> np.ndarray:
    axis = random_unit_vectors(rng, 1)[0]
    angle = math.radians(rng.uniform(0.0, max_angle_deg))
    return rotation_axis_angle(axis, angle)


def _knn(points: np.ndarray, k: int):
    from scipy.spatial import cKDTree
    tree = cKDTree(points)
    dist, idx = tree.query(points, k=k + 1)
    return dist[:, 1:], idx[:, 1:]


def _sensor_diag_cov(points: np.ndarray) -> np.ndarray:
    """diag(s^2, s^2, (2 s)^2) with s = mean distance to the 8 nearest neighbours."""
    dist, _ = _knn(points, 8)
    s = dist.mean(axis=1)
    C = np.zeros((points.shape[0], 3, 3))
    C[:, 0, 0] = s * s
    C[:, 1, 1] = s * s
    C[:, 2, 2] = 4.0 * s * s
    return C


def _knn_sample_cov(points: np.ndarray, lo: float = 1e-6, hi: float = 1e-2) -> np.ndarray:
    """8-NN sample covariance (point plus its 8 neighbours), eigenvalues clamped to [lo, hi]."""
    _, idx = _knn(points, 8)
    nb = np.concatenate([points[:, None, :], points[idx]], axis=1)   # (n, 9, 3)
    c = nb - nb.mean(axis=1, keepdims=True)
    C = np.einsum("nka,nkb->nab", c, c) / (nb.shape[1] - 1)
    w, V = np.linalg.eigh(C)
    w = np.clip(w, lo, hi)
    C = np.einsum("nab,nb,ncb->nac", V, w, V)
    return 0.5 * (C + np.transpose(C, (0, 2, 1)))


def _sphere_dirs(rng: np.random.Generator, n: int):
    v = random_unit_vectors(rng, n)
    theta = np.arccos(np.clip(v[:, 2], -1.0, 1.0))
    phi = np.arctan2(v[:, 1], v[:, 0])
    return v, theta, phi


def bumpy_sphere(rng: np.random.Generator, n: int) -> np.ndarray:
    """r = 1 + 0.1 sin(4 theta) cos(3 phi) on uniformly drawn directions."""
    v, theta, phi = _sphere_dirs(rng, n)
    r = 1.0 + 0.1 * np.sin(4.0 * theta) * np.cos(3.0 * phi)
    return v * r[:, None]


def harmonic_surface(rng: np.random.Generator, n: int, coeffs) -> np.ndarray:
    """Unit sphere plus a sum of real spherical harmonics (degree <= 6, amplitude 0.05)."""
    from scipy.special import sph_harm_y
    v, theta, phi = _sphere_dirs(rng, n)
    r = np.ones(n)
    for (l, m, a) in coeffs:
        Y = sph_harm_y(l, abs(m), theta, phi)
        real = np.sqrt(2.0) * (Y.real if m >= 0 else Y.imag) if m != 0 else Y.real
        r += a * real
    return v * r[:, None]


def _move(rng, S, max_angle_deg, tmax, noise):
    """Y = Rm S + tm + noise; returns Y and the ground truth mapping Y back onto X."""
    Rm = random_rotation(rng, max_angle_deg)
    tm = rng.uniform(-tmax, tmax, 3)
    Y = S @ Rm.T + tm + noise * rng.standard_normal(S.shape)
    R_G = Rm.T
    t_G = -Rm.T @ tm
    return Y, R_G, t_G


def workload0(trial: int = 0, n: int = 1000) -> Problem:
    """1000 x 1000 bumpy sphere, diag sensor-frame covariances from 8-NN spacing."""
    rng = rng_for(0, trial)
    X = bumpy_sphere(rng, n)
    S = bumpy_sphere(rng, n)
    Y, R_G, t_G = _move(rng, S, 60.0, 0.3, 0.01)
    return Problem(X, Y, _sensor_diag_cov(X), _sensor_diag_cov(Y), R_G, t_G, "sphere1k")


def _with_outliers(rng, P: np.ndarray, frac: float) -> np.ndarray:
    n_out = int(round(frac * P.shape[0]))
    lo, hi = P.min(axis=0), P.max(axis=0)
    c, h = 0.5 * (lo + hi), 0.5 * (hi - lo) * 1.2
    out = rng.uniform(c - h, c + h, (n_out, 3))
    keep = P[: P.shape[0] - n_out]
    return np.concatenate([keep, out], axis=0)


def workload1(trial: int = 0, n: int = 6000) -> Problem:
    """6000 x 6000 bumpy sphere, 10% of the points replaced by outliers, 8-NN sample covariances."""
    rng = rng_for(1, trial)
    X = _with_outliers(rng, bumpy_sphere(rng, n), 0.10)
    S = _with_outliers(rng, bumpy_sphere(rng, n), 0.10)
    Y, R_G, t_G = _move(rng, S, 60.0, 0.3, 0.01)
    return Problem(X, Y, _knn_sample_cov(X), _knn_sample_cov(Y), R_G, t_G, "sphere6k")


def workload2(trial: int = 0, n: int = 65536) -> Problem:
    """65536 x 65536 spherical-harmonic surface, noise 0.005, rotation <= 90 deg, t in [-0.5,0.5]^3."""
    rng = rng_for(2, trial)
    coeffs = []
    for _ in range(16):
        l = int(rng.integers(0, 7))
        m = int(rng.integers(-l, l + 1))
        coeffs.append((l, m, 0.05 * rng.uniform(-1.0, 1.0)))
    X = harmonic_surface(rng, n, coeffs)
    S = harmonic_surface(rng, n, coeffs)
    Y, R_G, t_G = _move(rng, S, 90.0, 0.5, 0.005)
    X += 0.005 * rng.standard_normal(X.shape)
    return Problem(X, Y, _knn_sample_cov(X), _knn_sample_cov(Y), R_G, t_G, "harmonic64k")


def so3_grid(rng: np.random.Generator, n: int) -> np.ndarray:
    """n well-spread rotations: super-Fibonacci quaternions with a seeded random offset rotation."""
    phi = math.sqrt(2.0)
    psi = 1.533751168755204288118041
    out = np.zeros((n, 3, 3))
    Q0 = random_rotation(rng, 180.0)
    for i in range(n):
        s = i + 0.5
        r = math.sqrt(s / n)
        R = math.sqrt(1.0 - s / n)
        a = 2.0 * math.pi * s / phi
        b = 2.0 * math.pi * s / psi
        w, x, y, z = r * math.sin(a), r * math.cos(a), R * math.sin(b), R * math.cos(b)
        out[i] = Q0 @ np.array([
            [1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)],
            [2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)],
            [2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)]])
    return out


def workload3(trial: int = 0, n_problems: int = 256, n_poses: int = 32,
              lo: int = 500, hi: int = 8000) -> list[Problem]:
    """n_problems independent bumpy-sphere problems with N, M iid uniform in [lo, hi]."""
    rng = rng_for(3, trial)
    probs = []
    for p in range(n_problems):
        n = int(rng.integers(lo, hi + 1))
        m = int(rng.integers(lo, hi + 1))
        X = bumpy_sphere(rng, n)
        S = bumpy_sphere(rng, m)
        Y, R_G, t_G = _move(rng, S, 60.0, 0.3, 0.01)
        probs.append(Problem(X, Y, _sensor_diag_cov(X), _sensor_diag_cov(Y), R_G, t_G, f"batch{p}"))
    return probs


def _range_view(rng, n_keep, boxes, spheres, view_R, view_t, camera=(640, 480, 525.0, 525.0, 319.5, 239.5)):
    """Ray-cast a box-and-sphere scene from a pinhole camera (W, H, fx, fy, cx, cy)."""
    W, H, fx, fy, cx, cy = camera
    u, v = np.meshgrid(np.arange(W), np.arange(H))
    dirs = np.stack([(u - cx) / fx, (v - cy) / fy, np.ones_like(u, dtype=np.float64)], axis=-1).reshape(-1, 3)
    z = np.full(dirs.shape[0], np.inf)
    o = view_t
    dw = dirs @ view_R.T
    for (c, r) in spheres:
        oc = o - c
        b = dw @ oc
        a = np.einsum("ij,ij->i", dw, dw)
        cc = oc @ oc - r * r
        disc = b * b - a * cc
        ok = disc >= 0
        s = np.where(ok, (-b - np.sqrt(np.where(ok, disc, 0))) / a, np.inf)
        s = np.where(s > 0, s, np.inf)
        z = np.minimum(z, s)
    for (lo, hi) in boxes:
        with np.errstate(divide="ignore", invalid="ignore"):
            t1 = (lo - o) / dw
            t2 = (hi - o) / dw
        tmin = np.nanmax(np.minimum(t1, t2), axis=1)
        tmax = np.nanmin(np.maximum(t1, t2), axis=1)
        hit = (tmax >= tmin) & (tmin > 0)
        z = np.minimum(z, np.where(hit, tmin, np.inf))
    valid = np.isfinite(z) & (z >= 0.5) & (z <= 4.0)
    idx = np.flatnonzero(valid)
    idx = rng.choice(idx, size=min(n_keep, idx.size), replace=False)
    zc = z[idx]
    P_cam = dirs[idx] * zc[:, None]
    sxy = 0.0015 * zc
    sz = 0.0028 * zc * zc
    C_cam = np.zeros((idx.size, 3, 3))
    C_cam[:, 0, 0] = sxy ** 2
    C_cam[:, 1, 1] = sxy ** 2
    C_cam[:, 2, 2] = sz ** 2
    P_cam = P_cam + rng.standard_normal(P_cam.shape) * np.stack([sxy, sxy, sz], axis=1)
    return P_cam, C_cam


def workload4(trial: int = 0, n: int = 300000) -> Problem:
    """Two depth-camera views of a random box-and-sphere scene, n points each, depth-dependent covariances."""
    rng = rng_for(4, trial)
    boxes, spheres = [], []
    for _ in range(6):
        c = np.array([rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0), rng.uniform(0.6, 3.0)])
        h = rng.uniform(0.1, 0.5, 3)
        boxes.append((c - h, c + h))
    for _ in range(4):
        c = np.array([rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0), rng.uniform(0.6, 3.0)])
        spheres.append((c, rng.uniform(0.2, 0.6)))
    # a back wall wide and near enough that every pixel of both views hits something within 4 m
    boxes.append((np.array([-10.0, -8.0, 3.5]), np.array([10.0, 8.0, 3.6])))
    Xc, XC = _range_view(rng, n, boxes, spheres, np.eye(3), np.zeros(3))
    Rv = random_rotation(rng, 15.0)
    tv = rng.uniform(-0.1, 0.1, 3)
    Yc, YC = _range_view(rng, n, boxes, spheres, Rv, tv)
    # camera-frame points of view 2 map to the world (= view 1 frame) by y_w = Rv y + tv
    return Problem(Xc, Yc, XC, YC, Rv, tv, "depth300k")


def _random_scene(rng, n_boxes=6, n_spheres=4, z=(0.6, 3.0), wall=None):
    """Axis-aligned boxes and spheres in front of the camera, optionally a back wall at depth `wall`."""
    boxes, spheres = [], []
    for _ in range(n_boxes):
        c = np.array([rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0), rng.uniform(*z)])
        h = rng.uniform(0.1, 0.5, 3)
        boxes.append((c - h, c + h))
    for _ in range(n_spheres):
        c = np.array([rng.uniform(-1.5, 1.5), rng.uniform(-1.0, 1.0), rng.uniform(*z)])
        spheres.append((c, rng.uniform(0.2, 0.6)))
    if wall is not None:
        boxes.append((np.array([-10.0, -8.0, wall]), np.array([10.0, 8.0, wall + 0.1])))
    return boxes, spheres


KINECT_V2 = (512, 424, 365.0, 365.0, 255.5, 211.5)


def kinect_like(trial: int = 0) -> Problem:
    """Stand-in for one two-sensor depth scene (the shape of the reference's 30 Kinect scenes:
    clouds cropped to the shared ~1.2 m working volume, N ~ U[3598, 5334] and M ~ U[463, 5159]
    points, isotropic "uncertainty" covariances c_i I with c_i in [1.3, 7.9]).

    12 boxes and 8 spheres fill a 1.2 m volume centred 1.8 m in front of camera 1 (the world
    frame).  Camera 2 orbits the volume's centre by a rotation of up to 30 deg about a random
    axis, plus a translation in [-0.1, 0.1]^3 m, so it sees the scene from another side.  Both
    are 512x424 depth cameras (f = 365 px).  Each view keeps its points inside the working
    volume, is subsampled, and expressed in its own camera frame; c_i grows geometrically
    with the point's depth from 1.3 at 0.5 m to 7.9 at 4 m.  Ground truth: R_G y + t_G is the
    world position of camera-2 point y."""
    rng = rng_for(5, trial)
    centre = np.array([0.0, 0.0, 1.8])
    boxes, spheres = [], []
    for _ in range(12):
        c = centre + rng.uniform(-0.45, 0.45, 3)
        h = rng.uniform(0.05, 0.2, 3)
        boxes.append((c - h, c + h))
    for _ in range(8):
        spheres.append((centre + rng.uniform(-0.45, 0.45, 3), rng.uniform(0.08, 0.25)))
    n = int(rng.integers(3598, 5335))
    m = int(rng.integers(463, 5160))
    Rv = random_rotation(rng, 30.0)
    tv = centre - Rv @ centre + rng.uniform(-0.1, 0.1, 3)

    def view(R, t, k):
        P, _ = _range_view(rng, 10 ** 9, boxes, spheres, R, t, KINECT_V2)
        world = P @ R.T + t
        keep = np.flatnonzero(np.all(np.abs(world - centre) <= 0.6, axis=1))
        keep = rng.choice(keep, size=min(k, keep.size), replace=False)
        P = P[keep]
        c = 1.3 * (7.9 / 1.3) ** np.clip((P[:, 2] - 0.5) / 3.5, 0.0, 1.0)
        return P, c[:, None, None] * np.eye(3)

    X, XC = view(np.eye(3), np.zeros(3), n)
    Y, YC = view(Rv, tv, m)
    return Problem(X, Y, XC, YC, Rv, tv, f"twoview{trial}")


def curve_shape(rng: np.random.Generator, n_bumps: int = 6, amp: float = 0.08):
    """A closed curve r(a) = 1 + sum_k c_k sin(k a + p_k), k = 1..n_bumps: returns (c, p)."""
    return rng.uniform(-amp, amp, n_bumps), rng.uniform(0.0, 2.0 * np.pi, n_bumps)


def curve_points(shape, a: np.ndarray):
    """Points of the curve at angles a, with the unit tangent at each."""
    c, ph = shape
    k = np.arange(1, len(c) + 1)
    r = 1.0 + np.sin(np.outer(a, k) + ph) @ c
    dr = np.cos(np.outer(a, k) + ph) @ (c * k)
    P = np.stack([r * np.cos(a), r * np.sin(a)], axis=1)
    T = np.stack([dr * np.cos(a) - r * np.sin(a), dr * np.sin(a) + r * np.cos(a)], axis=1)
    return P, T / np.linalg.norm(T, axis=1, keepdims=True)


def _tangent_cov(T: np.ndarray, s_t: float, s_n: float) -> np.ndarray:
    """Covariance s_t^2 t t^T + s_n^2 n n^T per point (t the tangent, n its normal)."""
    N = np.stack([-T[:, 1], T[:, 0]], axis=1)
    return s_t ** 2 * T[:, :, None] * T[:, None, :] + s_n ** 2 * N[:, :, None] * N[:, None, :]


def workload5(trial: int = 0, n: int = 65536) -> Problem:
    """2D: 65536 x 65536 samples (random angles, random order) of one closed curve, radius
    1 + six random sine bumps of amplitude <= 0.08; the moving cloud rotated by up to 90 deg,
    shifted in [-0.5, 0.5]^2, noise 0.005; covariances along the local tangent (sigma 0.01)
    and across it (0.004)."""
    rng = rng_for(5, trial)
    shape = curve_shape(rng)
    X, TX = curve_points(shape, rng.uniform(0.0, 2.0 * np.pi, n))
    S, TS = curve_points(shape, rng.uniform(0.0, 2.0 * np.pi, n))
    ang = rng.uniform(-np.pi / 2, np.pi / 2)
    Rm = np.array([[np.cos(ang), -np.sin(ang)], [np.sin(ang), np.cos(ang)]])
    tm = rng.uniform(-0.5, 0.5, 2)
    Y = S @ Rm.T + tm + 0.005 * rng.standard_normal(S.shape)
    XC = _tangent_cov(TX, 0.01, 0.004)
    YC = _tangent_cov(TS @ Rm.T, 0.01, 0.004)
    return Problem(X, Y, XC, YC, Rm.T, -Rm.T @ tm, "curve64k_2d")


WORKLOADS = {0: workload0, 1: workload1, 2: workload2, 4: workload4, 5: workload5}


# ---------------------------------------------------------------------------
# The simulation protocol of main_simulation.m:17-35 on a model (the reference's 2D_SHAPE_MODEL /
# 2D_Fish_MODEL contours and its 3D_SHAPE surface, tests/golden/sim_models.npz), seeded
# ---------------------------------------------------------------------------
def _radius(P: np.ndarray):
    """get_radius.m:4-21: the centroid and sqrt(mean squared distance to it) of (n, D) points."""
    mean = P.mean(axis=0)
    return mean, math.sqrt(float(((P - mean) ** 2).sum()) / len(P))


def _noise_and_sampling(rng, model: np.ndarray, R_G: np.ndarray, t_G: np.ndarray, noi: float, miss: float,
                        for_y: bool):
    """noise_and_sampling2D.m:1-95 / noise_and_sampling3D.m:1-120 for one of their two outputs:
    per model point an axis-aligned covariance diag(exp(fa r_a)) with r_a = |noi * randn| per
    axis (fa = 3.4657), the point moved by r_a * randn * radius along each axis, a contiguous
    occluded patch (the round(miss * M) points nearest a random model point) left out, and the
    rest kept with probability 0.9 (X) or 0.85 (Y); Y's points and covariances are then mapped by
    (R_G, t_G)."""
    fa = 3.4657
    M, D = model.shape
    occ = rng.integers(0, M)
    d2 = ((model - model[occ]) ** 2).sum(axis=1)
    occluded = np.zeros(M, bool)
    occluded[np.argsort(d2, kind="stable")[:int(round(miss * M))]] = True
    _, radius = _radius(model)
    r = np.abs(noi * rng.standard_normal((M, D)))
    moved = model + r * rng.standard_normal((M, D)) * radius
    keep = (rng.random(M) <= (0.85 if for_y else 0.9)) & ~occluded
    P = moved[keep]
    C = np.zeros((int(keep.sum()), D, D))
    for a in range(D):
        C[:, a, a] = np.exp(r[keep, a] * fa)
    if for_y:
        P = P @ R_G.T + t_G
        C = R_G @ C @ R_G.T
    return P, C


def _eul2rotm_zyx(z: float, y: float, x: float) -> np.ndarray:
    """Rotation from ZYX Euler angles in radians: Rz(z) Ry(y) Rx(x)."""
    cz, sz, cy, sy, cx, sx = math.cos(z), math.sin(z), math.cos(y), math.sin(y), math.cos(x), math.sin(x)
    Rz = np.array([[cz, -sz, 0.0], [sz, cz, 0.0], [0.0, 0.0, 1.0]])
    Ry = np.array([[cy, 0.0, sy], [0.0, 1.0, 0.0], [-sy, 0.0, cy]])
    Rx = np.array([[1.0, 0.0, 0.0], [0.0, cx, -sx], [0.0, sx, cx]])
    return Rz @ Ry @ Rx


def simulation(model: np.ndarray, trial: int = 0, rand_degree: float = 30.0, rand_noise: float = 0.1,
               rand_outliers: int | None = None, rand_miss_rate: float = 0.1, name: str = "") -> Problem:
    """One registration problem of the reference's simulation (produce_point_cloud.m:1-52 with
    main_simulation.m:19-22 / 31-34's ranges): a rotation by U[-30, 30] deg (2D), or by ZYX Euler
    angles each in U[-30, 30] deg (3D, eul2rotm), a translation in [-0.5, 0.5]^D, a noise level in
    [0, 0.1], up to 50 (2D) or 100 (3D) outliers (add_outliers.m: Gaussian around the model's
    centroid with its radius as deviation, drawn separately for X and Y) and an occlusion rate in
    [0, 0.1]; X and Y are sampled from the model independently (noise_and_sampling2D.m /
    noise_and_sampling3D.m).  Returned with the ground truth of produce_point_cloud.m:49-50, the
    pose that maps Y back onto X: R_G @ y + t_G ~ x.  model: (n, D) points."""
    model = np.asarray(model, dtype=np.float64)
    D = model.shape[1]
    if rand_outliers is None:
        rand_outliers = 50 if D == 2 else 100
    rng = rng_for(60 if D == 2 else 61, trial)
    if D == 2:
        deg = rand_degree * (2 * rng.random() - 1)
        c, s = math.cos(math.radians(deg)), math.sin(math.radians(deg))
        R = np.array([[c, -s], [s, c]])
    else:
        dx, dy, dz = (rand_degree * (2 * rng.random() - 1) for _ in range(3))
        R = _eul2rotm_zyx(math.radians(dz), math.radians(dy), math.radians(dx))
    noi = rand_noise * rng.random()
    n_out = int(round(rand_outliers * rng.random()))
    miss = rand_miss_rate * rng.random()
    t = (1 - 2 * rng.random(D)) * 0.5
    mean, radius = _radius(model)
    mx = np.concatenate([model, rng.standard_normal((n_out, D)) * radius + mean])
    my = np.concatenate([model, rng.standard_normal((n_out, D)) * radius + mean])
    X, X_C = _noise_and_sampling(rng, mx, R, t, noi, miss, False)
    Y, Y_C = _noise_and_sampling(rng, my, R, t, noi, miss, True)
    return Problem(X, Y, X_C, Y_C, R.T.copy(), -R.T @ t, name or f"sim{D}d_{trial}")
