"""The GPU bench drivers (bin/pac_bench): the reference's bench*.c command
line (verify|bench -t power -r runs), one driver per reference program, and
the t lists of bench{1,2,3}d.sh."""
import json
import os
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "c-permutation-avoiding-convolution_b200", "bin", "pac_bench")
DRIVERS = ["1d_forward_fft", "1d_backward_fft", "1d_convolution", "2d_forward_fft",
           "2d_backward_fft", "2d_convolution", "2d_convolution_anisotropic", "3d_forward_fft",
           "3d_backward_fft", "3d_convolution", "3d_convolution_anisotropic"]
# small powers: 1D 2^12, 2D 64 x 64 (anisotropic 2^12 x 4), 3D 16^3
# (anisotropic 2^8 x 4 x 4); every radix the reference runs at these sizes
SMALL_T = {"1d": 12, "2d": 6, "2d_a": 12, "3d": 4, "3d_a": 8}


def small_t(driver):
    key = driver[:2] + ("_a" if driver.endswith("anisotropic") else "")
    return SMALL_T[key]


def run(*args, timeout=300):
    return subprocess.run([BIN, *args], capture_output=True, text=True, timeout=timeout)


@pytest.fixture(scope="module")
def binary(lib):
    assert os.path.exists(BIN), "bin/pac_bench is built by the package Makefile"
    return BIN


def test_command_line(lib):
    """Usage, unknown drivers and modes fail with status 1 before any device
    work, as the reference's drivers do."""
    assert os.path.exists(BIN)
    r = run()
    assert r.returncode == 1 and "Usage" in r.stderr
    for d in DRIVERS:
        assert d in r.stderr
    assert run("4d_convolution", "bench").returncode == 1
    assert run("1d_convolution", "time").returncode == 1
    assert run("1d_convolution", "bench", "-x", "3").returncode == 1
    assert run("sweep", "5d").returncode == 1


def _rows(out):
    return [json.loads(line) for line in out.splitlines() if line.startswith("{")]


@pytest.mark.gpu
@pytest.mark.parametrize("driver", DRIVERS)
def test_verify_against_cpu_fft(binary, driver):
    t = small_t(driver)
    r = run(driver, "verify", "-t", str(t), "--json")
    assert r.returncode == 0, r.stderr
    rows = _rows(r.stdout)
    radices = {row["radix"] for row in rows}
    assert 2 in radices
    if t % 2 == 0:
        assert 4 in radices
    dims_n = {"1d": 2 ** t, "2d": 4 ** t, "3d": 8 ** t}[driver[:2]]
    if driver.endswith("anisotropic"):
        dims_n = 2 ** t * (4 if driver.startswith("2d") else 16)
    for row in rows:
        # values in [0, 1]: transforms and convolutions grow like n; FP64
        # error per element stays a few ulps of that
        assert row["max_error_vs_cpu_fft"] < 1e-13 * dims_n + 1e-12, row


@pytest.mark.gpu
@pytest.mark.parametrize("driver", ["1d_convolution", "2d_forward_fft", "3d_backward_fft"])
def test_bench_json(binary, driver):
    r = run(driver, "bench", "-t", str(small_t(driver)), "-r", "2", "--json")
    assert r.returncode == 0, r.stderr
    rows = _rows(r.stdout)
    paths = {row["path"] for row in rows}
    assert paths == {"fft.h, host buffers", "pac.h, device-resident"}
    assert all(row["mean_s"] > 0 for row in rows)


SWEEPS = {  # the t lists of the reference's bench1d.sh, bench2d.sh, bench3d.sh
    "1d": {d: [20, 22, 24, 26, 28] for d in DRIVERS[:3]},
    "2d": {**{d: [10, 11, 12, 13, 14] for d in DRIVERS[3:6]},
           "2d_convolution_anisotropic": [20, 22, 24, 26]},
    "3d": {**{d: [7, 8, 9] for d in DRIVERS[7:10]},
           "3d_convolution_anisotropic": [20, 22, 24]},
}


@pytest.mark.parametrize("which", sorted(SWEEPS))
def test_sweep_lists(lib, which):
    r = run("sweep", which, "--list")
    assert r.returncode == 0, r.stderr
    got = {}
    for row in _rows(r.stdout):
        got.setdefault(row["driver"], []).append(row["t"])
    assert got == SWEEPS[which]
