"""The kernels' small-matrix math (csrc/common.cuh, compiled here as host code
by nvcc) against numpy / scipy: polar rotation (Newton and SVD paths), the
3x3 / 2x2 rotation-variant SVD, the factorised GIMP weights and the
snow-projection skip test."""
import ctypes
import os
import shutil
import subprocess

import numpy as np
import pytest

import oracle as O
from conftest import REPO

HARNESS = os.path.join(REPO, "tests", "cuda_harness", "math_harness.cu")


@pytest.fixture(scope="module")
def h(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    out = str(tmp_path_factory.mktemp("harness") / "libmath_harness.so")
    subprocess.run([nvcc, "-O2", "-std=c++17", "--expt-relaxed-constexpr", "-Xcompiler", "-fPIC", "-shared",
                    "-I", os.path.join(REPO, "include"), HARNESS, "-o", out], check=True)
    return ctypes.CDLL(out)


def f32p(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def rand_F(rng, n, dim, spread):
    F = np.eye(dim) + rng.normal(0, spread, (n, dim, dim))
    Q = np.linalg.qr(rng.normal(size=(n, dim, dim)))[0]
    Q[:, :, 0] *= np.sign(np.linalg.det(Q))[:, None]  # proper rotations
    return (Q @ F).astype(np.float32)


@pytest.mark.parametrize("spread", [1e-3, 0.05, 0.3])
def test_polar_rotation_3d(h, spread):
    from scipy.linalg import polar
    rng = np.random.default_rng(1)
    F = rand_F(rng, 2000, 3, spread)
    F = F[np.linalg.det(F) > 0.05]
    R = np.zeros_like(F)
    h.h_polar_rot(3, f32p(F), f32p(R), len(F))
    ref = np.array([polar(f.astype(np.float64))[0] for f in F])
    assert np.abs(R - ref).max() < 2e-5


def test_newton_path_converges_near_rotations(h):
    rng = np.random.default_rng(2)
    F = rand_F(rng, 2000, 3, 0.02)  # the snow range: singular values near 1
    R = np.zeros_like(F)
    ok = np.zeros(len(F), np.int32)
    h.h_polar_newton3(f32p(F), f32p(R), ok.ctypes.data_as(ctypes.c_void_p), len(F))
    assert ok.all()
    np.testing.assert_allclose(np.einsum("nij,nkj->nik", R, R), np.broadcast_to(np.eye(3), R.shape), atol=2e-6)


def test_newton_rejects_inverted(h):
    F = np.diag([1.0, 1.0, -1.0]).astype(np.float32)[None]
    R = np.zeros_like(F)
    ok = np.zeros(1, np.int32)
    h.h_polar_newton3(f32p(F), f32p(R), ok.ctypes.data_as(ctypes.c_void_p), 1)
    assert ok[0] == 0


@pytest.mark.parametrize("dim", [2, 3])
def test_polar_rot_matches_oracle_stress_rotation(h, dim):
    """Inverted F included: R is the rotation of the rotation-variant SVD."""
    rng = np.random.default_rng(3)
    F = rand_F(rng, 500, dim, 0.6)
    R = np.zeros_like(F)
    h.h_polar_rot(dim, f32p(F), f32p(R), len(F))
    for f, r in zip(F, R):
        U, S, V = O.svd(f)
        if abs(S[-1]) < 1e-3 * abs(S[0]):
            continue  # rotation ill-defined
        np.testing.assert_allclose(r, U @ V.T, atol=5e-5)


@pytest.mark.parametrize("dim", [2, 3])
def test_svd(h, dim):
    rng = np.random.default_rng(4)
    A = rand_F(rng, 1000, dim, 0.5)
    U, S, V = np.zeros_like(A), np.zeros((len(A), dim), np.float32), np.zeros_like(A)
    h.h_svd(dim, f32p(A), f32p(U), f32p(S), f32p(V), len(A))
    rec = np.einsum("nij,nj,nkj->nik", U, S, V)
    assert np.abs(rec - A).max() < 5e-5
    assert np.all(np.linalg.det(U) > 0.999) and np.all(np.linalg.det(V) > 0.999)
    ref = np.linalg.svd(A.astype(np.float64), compute_uv=False)
    np.testing.assert_allclose(np.abs(S), ref, atol=5e-5)
    assert np.all(np.sign(S[:, -1]) == np.sign(np.linalg.det(A)))


def test_axis_weights_reproduce_reference_stencil(h):
    """Product of per-axis sums == the reference's sum of per-cell products
    (utils.py:18-42, adaptive_gimp.py:218-228, via the oracle in f64)."""
    rng = np.random.default_rng(5)
    for _ in range(200):
        tc = rng.uniform(-0.5, 0.5, 3)
        Wa = [np.zeros(3, np.float32) for _ in range(3)]
        Ga = [np.zeros(3, np.float32) for _ in range(3)]
        for d in range(3):
            h.h_axis_weights(ctypes.c_float(tc[d]), ctypes.c_float(0.5), f32p(Wa[d]), f32p(Ga[d]))
        ref = O.weight_stencil(tc, 0.5, f64=True)
        for k in range(27):
            n = (k % 3, (k // 3) % 3, k // 9)  # conv (1, 3, 9)
            w = Wa[0][n[0]] * Wa[1][n[1]] * Wa[2][n[2]] / 8.0
            g = np.array([Ga[0][n[0]] * Wa[1][n[1]] * Wa[2][n[2]], Wa[0][n[0]] * Ga[1][n[1]] * Wa[2][n[2]],
                          Wa[0][n[0]] * Wa[1][n[1]] * Ga[2][n[2]]]) / 4.0
            assert abs(w - ref[k, 0]) < 1e-6
            np.testing.assert_allclose(g, ref[k, 1:], atol=1e-6)


def test_axis_weights_half_match_general_form(h):
    """The closed form for radius 1/2 equals the clamped general form on
    t in [-0.5, 0.5] (to rounding)."""
    for t in np.linspace(-0.5, 0.5, 1001):
        W, G, Wh, Gh = (np.zeros(3, np.float32) for _ in range(4))
        h.h_axis_weights(ctypes.c_float(t), ctypes.c_float(0.5), f32p(W), f32p(G))
        h.h_axis_weights_half(ctypes.c_float(t), f32p(Wh), f32p(Gh))
        np.testing.assert_allclose(Wh, W, atol=4e-7)
        np.testing.assert_allclose(Gh, G, atol=4e-7)


@pytest.mark.parametrize("dim,spread", [(2, 0.3), (3, 0.004), (3, 0.02), (3, 0.05), (3, 0.3)])
def test_kirchhoff_stress_matches_oracle(h, dim, spread):
    """The P2G stress (series path near rotations, polar path elsewhere,
    inverted F included) against the oracle's SVD-based get_stress
    (utils.py:11-16) in f64, relative to the deviatoric part's size."""
    rng = np.random.default_rng(7)
    F = rand_F(rng, 1500, dim, spread)
    mu, la = 1000.0, 600.0
    tau = np.zeros_like(F)
    h.h_kirchhoff(dim, f32p(F), ctypes.c_float(mu), ctypes.c_float(la), f32p(tau), len(F))
    worst = 0.0
    for f, t in zip(F, tau):
        U, S, V = O.svd(f)
        if abs(S[-1]) < 1e-3 * abs(S[0]):
            continue  # rotation ill-defined
        ref = O.stress(f.astype(np.float64), mu, la, f64=True)
        scale = 2 * mu * np.abs(f - U @ V.T).max() * np.abs(f).max() + la * abs(np.linalg.det(f)) + 1e-3 * mu
        worst = max(worst, np.abs(t - ref).max() / scale)
    assert worst < 2e-5, worst


@pytest.mark.parametrize("dim", [2, 3])
def test_snow_skip_is_sound(h, dim):
    """Whenever the skip test passes, every singular value is inside the clamp
    interval and det F > 0, so the projection would not change F."""
    rng = np.random.default_rng(6)
    lo, hi = 1 - 2.5e-2, 1 + 7.5e-3
    F = rand_F(rng, 20000, dim, 0.004)
    out = np.zeros(len(F), np.int32)
    h.h_within(dim, f32p(F), ctypes.c_float(lo), ctypes.c_float(hi), out.ctypes.data_as(ctypes.c_void_p), len(F))
    s = np.linalg.svd(F.astype(np.float64), compute_uv=False)
    sel = out == 1
    assert sel.sum() > 1000
    assert np.all(s[sel] >= lo - 1e-6) and np.all(s[sel] <= hi + 1e-6)
    assert np.all(np.linalg.det(F[sel]) > 0)


@pytest.mark.parametrize("dim", [2, 3])
def test_corner_elements_match_elem_of(h, dim):
    """The per-axis corner indices of the binning's level search give the
    same element (and the same in-store answer) as elem_of / in_store for
    every corner, block boundaries and the store's edges included."""
    rng = np.random.default_rng(11)
    nb = 19  # 64 cells per axis + 3 halo blocks
    I0 = rng.integers(-7, 4 * nb - 1, (4000, dim)).astype(np.int32)
    I0[:64] = np.array([[3, 3, 3][:dim]] * 64) + rng.integers(-1, 1, (64, dim))  # around a block corner
    n, k = len(I0), 1 << dim
    idx, ok = np.zeros(n * k, np.uint32), np.zeros(n * k, np.int32)
    ref_idx, ref_ok = np.zeros(n * k, np.int64), np.zeros(n * k, np.int32)
    h.h_corners(dim, nb, I0.ctypes.data_as(ctypes.c_void_p), n, idx.ctypes.data_as(ctypes.c_void_p),
                ok.ctypes.data_as(ctypes.c_void_p), ref_idx.ctypes.data_as(ctypes.c_void_p),
                ref_ok.ctypes.data_as(ctypes.c_void_p))
    np.testing.assert_array_equal(ok, ref_ok)
    assert ok.sum() > n * k // 2 and (ok == 0).sum() > 0
    np.testing.assert_array_equal(idx[ok == 1].astype(np.int64), ref_idx[ok == 1])
