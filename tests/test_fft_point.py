"""The bench's cuFFT comparison point for the density solve (bench.fft_density_solve) against
the engine's own definition of the solve, evaluated directly here in double: the forward 2-D
DCT with its scaling, the spectral step, and the DST-DCT / DCT-DST inverses with the k = 0
sine term taken as (-1)^n (the basis matrices of csrc/kernels/poisson.cu, build_basis).
CPU, float64: the FFT forms are the same sums to rounding."""
import numpy as np
import pytest
import torch

import bench


def _cos(n):
    return np.cos(np.pi * np.outer(np.arange(n), np.arange(n) + 0.5) / n)  # [k][j]


def _sin(n):
    k = np.arange(n)[:, None]
    return np.where(k == 0, (-1.0) ** np.arange(n)[None, :], np.sin(np.pi * k * (np.arange(n)[None, :] + 0.5) / n))


def _scale(n):
    return np.where(np.arange(n) == 0, 1.0 / n, 2.0 / n)


@pytest.mark.parametrize("nx,ny", [(32, 32), (32, 16), (12, 10), (7, 9)])
def test_fft_solve_matches_the_basis_form(nx, ny):
    rng = np.random.default_rng(nx * 100 + ny)
    rho = rng.random((nx, ny)) * 1.5
    wx = np.pi * np.arange(nx) / nx
    wy = np.pi * np.arange(ny) / ny * (nx / ny)
    A = (_scale(nx)[:, None] * _cos(nx)) @ rho @ (_scale(ny)[:, None] * _cos(ny)).T
    d = wx[:, None] ** 2 + wy[None, :] ** 2
    d[0, 0] = 1.0
    P = A / d
    P[0, 0] = 0.0
    ex = _sin(nx).T @ (P * wx[:, None]) @ _cos(ny)
    ey = _cos(nx).T @ (P * wy[None, :]) @ _sin(ny)
    gx, gy = bench.fft_density_solve(torch.from_numpy(rho), torch.from_numpy(wx), torch.from_numpy(wy))
    assert np.abs(gx.numpy() - ex).max() <= 1e-12 * np.abs(ex).max()
    assert np.abs(gy.numpy() - ey).max() <= 1e-12 * np.abs(ey).max()
