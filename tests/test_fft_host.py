"""The PME mesh transforms' line FFT (pygcmc_b200/csrc/fft.cuh) against
numpy's FFT, run on the host: the Stockham radix-2/3 stages that the mesh
kernels execute are __host__ __device__ code, compiled here into a small host
program (tests/fft_line_check.cu)."""
import os
import subprocess

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def fft_bin(tmp_path_factory):
    out = str(tmp_path_factory.mktemp("fft") / "fft_line_check")
    subprocess.check_call(["nvcc", "-std=c++17", "-O2", "-o", out, os.path.join(HERE, "fft_line_check.cu")])
    return out


def run_lines(binary, cases):
    inp = []
    for n, sign, x in cases:
        inp.append(f"{n} {sign}")
        inp.extend(f"{float(v.real)!r} {float(v.imag)!r}" for v in x)
    res = subprocess.run([binary], input="\n".join(inp) + "\n", capture_output=True, text=True, check=True)
    vals = np.array([[float(t) for t in line.split()] for line in res.stdout.split("\n") if line.strip()])
    out, pos = [], 0
    for n, _, _ in cases:
        out.append(vals[pos:pos + n, 0] + 1j * vals[pos:pos + n, 1])
        pos += n
    return out


def test_line_fft_matches_numpy(fft_bin):
    g = np.random.default_rng(7)
    sizes = [1, 2, 3, 4, 6, 8, 9, 12, 16, 18, 24, 27, 32, 48, 64, 96, 128, 144, 192, 216, 256]
    cases = []
    for n in sizes:
        for sign in (-1, 1):
            cases.append((n, sign, g.normal(size=n) + 1j * g.normal(size=n)))
    outs = run_lines(fft_bin, cases)
    for (n, sign, x), y in zip(cases, outs):
        ref = np.fft.fft(x) if sign < 0 else np.fft.ifft(x) * n  # unnormalised inverse
        err = np.abs(y - ref).max() / max(1.0, np.abs(ref).max())
        assert err < 1e-13, (n, sign, err)


def test_real_mesh_round_trip_convention(fft_bin):
    """A real row through the forward transform, its half spectrum extended by
    Hermitian symmetry and the inverse transform gives n times the row (the
    rows passes of the mesh transform)."""
    g = np.random.default_rng(3)
    n = 96
    x = g.normal(size=n)
    (X,) = run_lines(fft_bin, [(n, -1, x.astype(complex))])
    half = X[: n // 2 + 1]
    full = np.concatenate([half, np.conj(half[1:n - n // 2][::-1])])
    (y,) = run_lines(fft_bin, [(n, 1, full)])
    assert np.abs(y.real / n - x).max() < 1e-13
