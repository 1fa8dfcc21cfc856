"""CPU tests of the host side: the C-ABI library loads and exports every
symbol include/airt.h declares, argument errors come back as status codes,
and the host tables/relaxation rules agree with the oracle."""
import ctypes as C
import os
import re

import numpy as np
import pytest

import airtoolsii_b200 as airt
from airtoolsii_b200 import _lib, solvers, testprobs
from oracle import airt_oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    txt = open(os.path.join(ROOT, "include", "airt.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(airt_\w+)\s*\(", txt)))


def test_library_exports_every_declared_symbol():
    names = _declared()
    assert len(names) >= 18
    L = C.CDLL(_lib.LIB_PATH)
    for nm in names:
        assert hasattr(L, nm), nm
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)
    assert _lib.lib().airt_version() >= 10000


def test_bad_csc_is_rejected_without_a_device():
    L = _lib.lib()
    h = C.c_void_p()
    jc = np.array([0, 2, 1], np.uint64)          # decreasing column starts
    ir = np.array([0, 1], np.uint64)
    pr = np.array([1.0, 2.0])
    st = L.airt_problem_from_csc(2, 2, _lib.u64ptr(jc), _lib.u64ptr(ir), _lib.dptr(pr), C.byref(h))
    assert st == _lib.AIRT_ERR_ARG
    assert b"nondecreasing" in L.airt_last_error()
    jc = np.array([1, 2, 2], np.uint64)
    assert L.airt_problem_from_csc(2, 2, _lib.u64ptr(jc), _lib.u64ptr(ir), _lib.dptr(pr),
                                   C.byref(h)) == _lib.AIRT_ERR_ARG
    assert L.airt_problem_from_csc(2, 2, None, None, None, C.byref(h)) == _lib.AIRT_ERR_ARG


def test_null_handle_calls_fail_cleanly():
    L = _lib.lib()
    x = np.zeros(3)
    assert L.airt_apply(None, _lib.dptr(x), _lib.dptr(x), 0) == _lib.AIRT_ERR_ARG
    assert L.airt_problem_size(None, None, None, None) == _lib.AIRT_ERR_ARG
    assert L.airt_profile_read(None, 0, None, None) == _lib.AIRT_ERR_ARG


def test_parallel_tables_match_oracle():
    for N, theta, p, d in [(64, None, None, None), (512, np.arange(360) * 0.5, 724, None),
                           (15, np.arange(0.0, 180.0, 7.5), 21, 18.5)]:
        a = testprobs.parallel_tables(N, theta, p, d)
        b = O.parallel_geometry(N, theta, p, d)
        for u, v in zip(a, b):
            np.testing.assert_array_equal(np.asarray(u), np.asarray(v))


def test_fan_tables_match_oracle():
    for N, theta, p in [(32, None, None), (1024, np.arange(720) * 0.5, 1448), (20, None, 27)]:
        a = testprobs.fan_tables(N, theta, p)
        b = O.fan_geometry(N, theta, p)
        for u, v in zip(a, b):
            np.testing.assert_array_equal(np.asarray(u), np.asarray(v))


def test_shepplogan_matches_oracle():
    for N in (16, 33, 64):
        np.testing.assert_array_equal(testprobs.phantomgallery("shepplogan", N).ravel(order="F"),
                                      O.shepplogan(N))


def test_seismic_tables_and_tectonic_match_oracle():
    for N, s, p in [(64, None, None), (10, 3, 7), (33, 1, 2), (512, None, None)]:
        a = testprobs.seismic_tables(N, s, p)
        b = O.seismic_geometry(N, s, p)
        assert a[:2] == b[:2]
        for u, v in zip(a[2:], b[2:]):
            np.testing.assert_array_equal(u, v)
    for N in (10, 13, 64, 101, 256):
        np.testing.assert_array_equal(testprobs.phantomgallery("tectonic", N), O.tectonic(N))
    with pytest.raises(ValueError):
        testprobs.tectonic(6)
    with pytest.raises(ValueError):
        testprobs.seismic_tables(8, [2, 3])


def test_sphere_tables_match_oracle():
    for N, ang, nc in [(16, None, None), (33, [0.0, 45.0, 97.5], 7), (128, None, None)]:
        t = testprobs.sphere_tables(N, ang, nc)
        angles, nc_, radii, nphi, dphi, center, dx = O.sphere_geometry(N, ang, nc)
        ck, sk = O.sphere_circle_tables(nphi, dphi)
        assert t[1] == nc_
        for u, v in zip(t[:1] + t[2:], (angles, O.cosd(angles), O.sind(angles), radii, nphi, ck, sk)):
            np.testing.assert_array_equal(u, v)
    x = np.array([-2.5, -1.5, -0.5, 0.5, 1.5, 2.4999999999999996, 0.49999999999999994, 3.0])
    np.testing.assert_array_equal(testprobs._round_half_away(x), [-3, -2, -1, 1, 2, 2, 0, 3])
    np.testing.assert_array_equal(O.mround_array(x), [-3, -2, -1, 1, 2, 2, 0, 3])


def test_fbp_kernel_is_the_filtered_impulse_response():
    """Circular convolution with fbp_kernel equals fbp.m's zero-pad / fft /
    filter / ifft / crop of one projection, for every filter."""
    from airtoolsii_b200 import analytic as F
    rng = np.random.default_rng(4)
    for nr in (17, 91, 130):
        col = rng.standard_normal(nr)
        for name in ("ram-lak", "shepp-logan", "cosine", "hamming", "hann"):
            h = F.fbp_kernel(nr, name)
            order = h.size
            assert order == max(64, 2 ** int(np.ceil(np.log2(2 * nr))))
            direct = np.array([sum(h[(i - j) % order] * col[j] for j in range(nr)) for i in range(nr)])
            pad = np.zeros(order)
            pad[:nr] = col
            ref = np.real(np.fft.ifft(np.fft.fft(pad) * F.fbp_filter(nr, name)))[:nr]
            np.testing.assert_allclose(direct, ref, rtol=1e-12, atol=1e-12)
    with pytest.raises(ValueError):
        F.fbp_filter(10, "bogus")


def test_random_ellipses_range_and_determinism():
    x1 = testprobs.random_ellipses(48, 10, seed=5)
    x2 = testprobs.random_ellipses(48, 10, seed=5)
    assert np.array_equal(x1, x2) and x1.min() >= 0 and x1.max() <= 1 and x1.max() > 0


@pytest.mark.parametrize("rule", ["psi1", "psi1mod", "psi2", "psi2mod"])
def test_relaxation_tables_match_oracle(rule):
    kind, _, tab = solvers._relax_sirt(rule, 0.7, 40)
    ref, casel, _, _ = O.calc_relaxpar_sirt(rule, 0.7, 40, None, 10)
    assert kind == casel == 3
    np.testing.assert_array_equal(tab, ref)


def test_default_and_user_relaxpar():
    kind, lam, _ = solvers._relax_sirt(None, 2.0, 10)
    assert kind == 1 and lam == 1.9 / 2.0
    with pytest.warns(UserWarning):
        solvers._relax_sirt(2.5, 1.0, 10)
    with pytest.raises(ValueError):
        solvers._relax_sirt("bogus", 1.0, 10)


def test_randk_stream_matches_oracle_stream():
    rng = np.random.default_rng(1)
    normAi = rng.random(50) ** 4
    normAi[[3, 7]] = 0
    rows, lam_rows = solvers._randk_stream(normAi, 0.0, 3, seed=9)
    st = O.RandStream(9)
    I = np.flatnonzero(normAi > 0)
    for k in range(3):
        ri, ii = O.art_sweep_rows(I, normAi, True, st, normAi.size)
        np.testing.assert_array_equal(rows[k], ri)
        np.testing.assert_array_equal(lam_rows[k], ii)


def test_bench_reference_arm_json_contract():
    """bench.py --impl reference (the CPU restatement timed on the host) prints
    one JSON line with the contract's keys (N=48 contract-check case), and the
    process that runs it imports no part of the product: neither the
    airtoolsii_b200 package nor a mapping of libairt.so."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    probe = ("import sys, runpy\n"
             "sys.argv = ['bench.py', '--impl', 'reference', '--tiny', '--steps', '1', '--warmup', '3']\n"
             "runpy.run_path('bench.py', run_name='__main__')\n"
             "maps = open('/proc/self/maps').read()\n"
             "print('PRODUCT_LOADED', int('airtoolsii_b200' in sys.modules or 'libairt' in maps))\n")
    out = subprocess.run([sys.executable, "-c", probe], capture_output=True, text=True,
                         timeout=300, cwd=root)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = out.stdout.strip().splitlines()
    assert lines[-1] == "PRODUCT_LOADED 0", lines[-1]
    line = json.loads(lines[-2])
    for key in ("metric", "value", "unit", "n_gpus", "steps", "warmup", "ms_per_step",
                "higher_is_better", "scaling", "vs_baseline", "dtype", "data", "config",
                "cpu_baseline", "e2e"):
        assert key in line, key
    assert line["impl"] == "reference" and line["value"] > 0 and line["warmup"] >= 3
    assert line["e2e"]["h2d_bytes_per_step"] == 0 and line["e2e"]["d2h_bytes_per_step"] == 0
    assert line["cpu_baseline"]["kind"] in ("port", "reference") and line["cpu_baseline"]["cores"] >= 1
    assert "workload" in line["config"]


def test_oracle_data_generators_match_product():
    """The CPU benchmark arm draws phantom and noise from the oracle's copies of
    the generators; they give the same arrays as the product's for a seed."""
    x1 = testprobs.random_ellipses(40, 12, seed=77)
    x2 = O.random_ellipses(40, 12, seed=77)
    np.testing.assert_array_equal(x1, x2)
    b1, e1 = testprobs.add_noise(x1 * 3.0, 0.02, seed=78)
    b2, e2 = O.add_noise(x2 * 3.0, 0.02, seed=78)
    np.testing.assert_array_equal(b1, b2)
    assert e1 == e2
