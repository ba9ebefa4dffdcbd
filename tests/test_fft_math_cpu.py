"""The identities the FFT form of the transform (eisenjoch_b200/csrc/fft.cu)
is built on, checked in FP64 against the DCT matrices of the GEMM forms
(the linear maps of density.rs:96-166, rustdct conventions):

  DCT-II  X[k] = sum_n x[n] cos(pi k (n + 1/2) / N)
          = Re(e^{-i pi k / 2N} V[k]),  V = FFT(v),  v[m] = x[2m], v[N-1-m] = x[2m+1]
  C3      x[n] = sum_k c_k X[k] cos(pi k (n + 1/2) / N),  c_0 = 1/2
          x[2m] = v[m], x[2m+1] = v[N-1-m],  v = sum_k V[k] e^{2 pi i k m / N},
          V[0] = X[0]/2, V[k] = e^{i pi k / 2N} (X[k] - i X[N-k]) / 2
  S3      x[n] = sum_k d_k X[k] sin(pi (k+1)(n + 1/2) / N) = (-1)^n C3(X reversed)[n]
  SG      x[n] = -sum_k X[k] sin(pi k (n + 1/2) / N) = -(-1)^n C3(Y)[n],  Y[0] = 0, Y[k] = X[N-k]

and the packing of two real transforms into one complex FFT (two real
inputs split by conjugate symmetry; two real outputs as real and imaginary
parts).  No GPU: the kernels themselves are checked against the oracle by
tests/test_gpu_fft.py."""

import numpy as np
import pytest


def mats(N):
    k = np.arange(N)[:, None]
    n = np.arange(N)[None, :]
    th = np.pi * k * (n + 0.5) / N
    c = np.ones(N)
    c[0] = 0.5
    d = np.ones(N)
    d[N - 1] = 0.5
    dct2 = np.cos(th)  # [k][n]
    c3 = (np.cos(th) * c[:, None]).T  # [n][k]
    s3 = (np.sin(np.pi * (k + 1) * (n + 0.5) / N) * d[:, None]).T
    sg = (-np.sin(th)).T
    return dct2, c3, s3, sg


def reorder(x):
    N = len(x)
    v = np.empty(N, x.dtype)
    v[: N // 2] = x[0::2]
    v[N // 2:] = x[1::2][::-1]
    return v


def unreorder(v):
    N = len(v)
    x = np.empty(N, v.dtype)
    x[0::2] = v[: N // 2]
    x[1::2] = v[::-1][: N // 2]
    return x


def dct2_fft(x):
    N = len(x)
    V = np.fft.fft(reorder(x))
    return np.real(np.exp(-1j * np.pi * np.arange(N) / (2 * N)) * V)


def c3_V(X):
    N = len(X)
    k = np.arange(1, N)
    V = np.empty(N, complex)
    V[0] = X[0] / 2
    V[1:] = 0.5 * (X[1:] - 1j * X[N - k]) * np.exp(1j * np.pi * k / (2 * N))
    return V


def c3_fft(X):
    N = len(X)
    return unreorder(np.real(np.fft.ifft(c3_V(X)) * N))


@pytest.mark.parametrize("N", [16, 32, 64, 512])
def test_line_transforms(N):
    rng = np.random.default_rng(N)
    x, X = rng.standard_normal(N), rng.standard_normal(N)
    dct2, c3, s3, sg = mats(N)
    n = np.arange(N)
    alt = (-1.0) ** n
    Y = np.zeros(N)
    Y[1:] = X[N - np.arange(1, N)]
    tol = 1e-12 * N
    assert np.abs(dct2_fft(x) - dct2 @ x).max() <= tol
    assert np.abs(c3_fft(X) - c3 @ X).max() <= tol
    assert np.abs(alt * c3_fft(X[::-1]) - s3 @ X).max() <= tol
    assert np.abs(-alt * c3_fft(Y) - sg @ X).max() <= tol


@pytest.mark.parametrize("N", [16, 128])
def test_two_real_transforms_per_fft(N):
    rng = np.random.default_rng(N + 1)
    a, b = rng.standard_normal(N), rng.standard_normal(N)
    dct2, c3, _, _ = mats(N)
    k = np.arange(N)
    q = np.exp(-1j * np.pi * k / (2 * N))
    # forward: one FFT of the two reordered lines as real and imaginary parts
    Z = np.fft.fft(reorder(a) + 1j * reorder(b))
    Zc = np.conj(Z[(N - k) % N])
    Va, Vb = (Z + Zc) / 2, (Z - Zc) / 2j
    assert np.abs(np.real(q * Va) - dct2 @ a).max() <= 1e-12 * N
    assert np.abs(np.real(q * Vb) - dct2 @ b).max() <= 1e-12 * N
    # inverse: one FFT of V_a + i V_b; the outputs are its real and imaginary parts
    v = np.fft.ifft(c3_V(a) + 1j * c3_V(b)) * N
    assert np.abs(unreorder(np.real(v)) - c3 @ a).max() <= 1e-12 * N
    assert np.abs(unreorder(np.imag(v)) - c3 @ b).max() <= 1e-12 * N
