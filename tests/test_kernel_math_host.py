"""The device arithmetic of the LBM collision (mpm_lbm_b200/csrc/d3q19.cuh)
and of the FP64 polar rotation (csrc/polar3.cuh), compiled as host C++,
against the CPU oracle (dense-matrix restatement of fluid.py:398-413)."""

import ctypes
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as orc

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(ROOT, "mpm_lbm_b200", "csrc")

SRC = r"""
#include "d3q19.cuh"
#include "polar3.cuh"
extern "C" void host_collide(const float* F, float rho, const float* u, const float* A, float s_v, float s_o, float* out) {
  const fsi::MrtK K = fsi::make_mrt_k(s_v, s_o);
  fsi::mrt_collide(F, rho, u[0], u[1], u[2], A[0], A[1], A[2], K, out);
}
extern "C" void host_collide_unforced(const float* F, float rho, const float* u, float s_v, float s_o, float* out) {
  const fsi::MrtK K = fsi::make_mrt_k(s_v, s_o);
  fsi::mrt_collide<false>(F, rho, u[0], u[1], u[2], 0.f, 0.f, 0.f, K, out);
}
extern "C" void host_moments(const float* F, float* m) { fsi::moments0(F, m[0], m[1], m[2], m[3]); }
extern "C" void host_polar(const double* F, double* R) { fsi::polar_rotation_d(F, R); }
extern "C" void host_polar_jacobi(const double* F, double* R) { fsi::polar_rotation_jacobi_d(F, R); }
extern "C" int host_polar_newton(const double* F, double* R) { return fsi::polar_rotation_newton_d(F, R) ? 1 : 0; }
"""


@pytest.fixture(scope="module")
def hostlib(tmp_path_factory):
    d = tmp_path_factory.mktemp("hostmath")
    src = d / "m.cpp"
    src.write_text(SRC)
    so = d / "libm.so"
    subprocess.run(["g++", "-O2", "-std=c++17", "-shared", "-fPIC", "-I", CSRC, str(src), "-o", str(so)], check=True)
    return ctypes.CDLL(str(so))


def P(a):
    return a.ctypes.data_as(ctypes.c_void_p)


@pytest.mark.parametrize("collision", ["mrt", "bgk"])
def test_fast_collision_equals_dense_reference(hostlib, collision):
    rng = np.random.default_rng(1)
    n = 64
    lbm = orc.OracleLBM(n, 1, 1, niu=1.0 / 30.0, relaxation_semantics="standard_lattice_kinematic_viscosity",
                        force=(1e-5, -3e-6, 2e-6), collision=collision, dtype=np.float64)
    lbm.init_simulation()
    w = orc.W
    F = (w[None, :] * (1 + 0.05 * rng.standard_normal((n, 19)))).reshape(n, 1, 1, 19)
    lbm.F[...] = F
    lbm.rho[...] = 1 + 0.01 * rng.standard_normal((n, 1, 1))
    lbm.v[...] = 0.03 * rng.standard_normal((n, 1, 1, 3))
    lbm.cell_force[...] = 1e-4 * rng.standard_normal((n, 1, 1, 3))
    lbm.colission()
    s = np.array(lbm.p.S[:])
    s_v, s_o = s[1], s[4]
    out = np.zeros(19, np.float32)
    for c in range(n):
        Fc = lbm.F[c, 0, 0].astype(np.float32)
        u = lbm.v[c, 0, 0].astype(np.float32)
        A = (np.array(lbm.p.force[:]) + lbm.cell_force[c, 0, 0]).astype(np.float32)
        hostlib.host_collide(P(Fc), ctypes.c_float(lbm.rho[c, 0, 0]), P(u), P(A), ctypes.c_float(s_v),
                             ctypes.c_float(s_o), P(out))
        np.testing.assert_allclose(out, lbm.f[c, 0, 0], rtol=2e-6, atol=3e-8)


def test_moments(hostlib):
    rng = np.random.default_rng(2)
    F = rng.random(19).astype(np.float32)
    m = np.zeros(4, np.float32)
    hostlib.host_moments(P(F), P(m))
    np.testing.assert_allclose(m[0], F.sum(), rtol=1e-6)
    np.testing.assert_allclose(m[1:], F @ orc.E.astype(np.float32), rtol=1e-5, atol=1e-6)


def test_polar_rotation_matches_oracle(hostlib):
    rng = np.random.default_rng(3)
    L = orc.lib()
    for t in range(300):
        F = np.eye(3) + 0.5 * rng.standard_normal((3, 3))
        if t == 0:
            F = np.diag([1.2, -0.8, 1.0])
        if t == 1:
            F = np.eye(3)
        R1, R2 = np.zeros(9), np.zeros(9)
        hostlib.host_polar(P(F.reshape(-1).copy()), P(R1))
        L.orc_polar_rotation(P(F.reshape(-1).copy()), P(R2))
        np.testing.assert_allclose(R1, R2, atol=1e-10)


def test_polar_newton_agrees_with_jacobi(hostlib):
    """The Newton fast path and the Jacobi/QR path give the same proper rotation
    wherever Newton applies (det F > 0), including strongly stretched and nearly
    singular gradients; inverted gradients are left to the Jacobi path."""
    hostlib.host_polar_newton.restype = ctypes.c_int
    rng = np.random.default_rng(11)
    used = 0
    for t in range(2000):
        A = rng.standard_normal((3, 3))
        Q, _ = np.linalg.qr(A)
        Q *= np.sign(np.linalg.det(Q))
        s = np.exp(rng.uniform(-6 if t % 4 == 0 else -1, 1, 3))
        V, _ = np.linalg.qr(rng.standard_normal((3, 3)))
        F = Q @ np.diag(s) @ V.T
        if t % 7 == 0:
            F = F @ np.diag([1, 1, -1])  # inverted
        R1, R2 = np.zeros(9), np.zeros(9)
        ok = hostlib.host_polar_newton(P(F.reshape(-1).copy()), P(R1))
        hostlib.host_polar_jacobi(P(F.reshape(-1).copy()), P(R2))
        if np.linalg.det(F) <= 0:
            assert ok == 0
            continue
        assert ok == 1, F
        used += 1
        np.testing.assert_allclose(R1, R2, atol=1e-9)
        R = R1.reshape(3, 3)
        np.testing.assert_allclose(R @ R.T, np.eye(3), atol=1e-12)
        # the polar factor itself: R = F (F^T F)^-1/2
        w, U = np.linalg.eigh(F.T @ F)
        Rref = F @ U @ np.diag(w ** -0.5) @ U.T
        np.testing.assert_allclose(R, Rref, atol=1e-6)
    assert used > 1500


def test_unforced_collision_equals_forced_with_zero_force(hostlib):
    """mrt_collide<false> (no Guo term evaluated) gives the same populations as
    the forced form with a zero force, bit for bit."""
    rng = np.random.default_rng(21)
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)
    for _ in range(200):
        F = (w * (1.0 + 0.05 * rng.standard_normal(19))).astype(np.float32)
        u = (0.05 * rng.standard_normal(3)).astype(np.float32)
        rho = np.float32(F.sum())
        A = np.zeros(3, np.float32)
        a, b = np.zeros(19, np.float32), np.zeros(19, np.float32)
        hostlib.host_collide(P(F), ctypes.c_float(rho), P(u), P(A), ctypes.c_float(1 / 0.6),
                             ctypes.c_float(1.4), P(a))
        hostlib.host_collide_unforced(P(F), ctypes.c_float(rho), P(u), ctypes.c_float(1 / 0.6),
                                      ctypes.c_float(1.4), P(b))
        np.testing.assert_array_equal(a, b)


def test_population_block_order_matches_the_device_index():
    """pop_blocks (the host writer's conversion) puts population s of cell i
    at (i / 32) * 608 + s * 32 + i % 32, the element index the kernels use,
    and i + (i >> 5) * 576 + 32 s is that index in the form the kernels
    compute it."""
    import torch

    from mpm_lbm_b200.lbm import pop_blocks

    pitch = 256
    planes = torch.arange(19 * pitch, dtype=torch.float32).reshape(19, pitch)  # value = s * pitch + i
    flat = pop_blocks(planes).reshape(-1)
    for s in (0, 1, 7, 18):
        for i in (0, 1, 31, 32, 33, 100, 255):
            idx = (i // 32) * 608 + s * 32 + i % 32
            assert idx == i + (i >> 5) * 576 + 32 * s
            assert int(flat[idx]) == s * pitch + i
