"""CPU checks of the oracle: FFT shim against numpy, the C restatement
against the unmodified reference (oracle/_ref) and the committed golden
fixtures, and known-answer tests from the lattice geometry."""
import glob
import json
import os

import numpy as np
import pytest

from _cases import fields, field_args, rel_err

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden")


@pytest.mark.parametrize("n", [8, 16, 24, 32, 30])
def test_shim_fft_matches_numpy(ora, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal((n, n, n))
    got = ora.ora_forward(n, 0, x)
    ref = np.fft.fftn(x)
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def test_shim_phase_only(ora):
    n = 16
    x = np.random.default_rng(3).standard_normal((n, n, n))
    got = ora.ora_forward(n, 0, x, use_only_phase=1)
    ref = np.fft.fftn(x)
    ref = ref / np.abs(ref)
    assert np.abs(got - ref).max() <= 1e-13


def test_xhi_dens_composition(ora):
    n = 16
    d, x = fields(n, 100.0)
    dd, xx = field_args(2, d, x)
    got = ora.ora_forward(n, 2, dd, xx)
    ref = np.fft.fftn(dd.astype(np.float64) * (1.0 - xx.astype(np.float64)))
    assert np.abs(got - ref).max() <= 1e-13 * np.abs(ref).max()


def _brute_triangles(m1, m2, m3, n):
    """#{(a,b,c) in S1 x S2 x S3 : a+b+c = 0 mod n} by direct convolution."""
    f = lambda m: m.astype(np.float64)
    c12 = np.real(np.fft.ifftn(np.fft.fftn(f(m1)) * np.fft.fftn(f(m2)))) * 1.0
    # c12[q] = #{a+b = q}; need q = -c
    neg = np.roll(np.flip(f(m3), axis=(0, 1, 2)), 1, axis=(0, 1, 2))
    return float(np.rint((c12 * neg).sum()))


@pytest.mark.parametrize("kb", [0, 2, 3])
def test_npoly_is_lattice_triangle_count(ora, kb):
    n, box = 16, 100.0
    p = ora.RunParams(grid_size=n, box_size=box, which_field=0, n=3, equilateral=0,
                      k1=3.0 * 2 * np.pi / box, k2=4.0 * 2 * np.pi / box, num_values=4,
                      kbinning=kb, dcos_theta=0.3)
    d, _ = fields(n, box)
    r = ora.ora_run(p, d)
    L = float(np.float32(box))
    for i in range(len(r.k)):
        kinds = {0: (0, 0, 0), 2: (0, 0, 1), 3: (2, 2, 3)}[kb]
        masks = []
        for leg in range(3):
            masks.append(ora.ora_filter(n, kinds[leg], r.kpoly[i, leg], r.kmin[i, leg],
                                        r.kmax[i, leg], 1.0, L))
        assert r.npoly[i] == pytest.approx(_brute_triangles(*masks, n), abs=1e-6)


def test_power_spectrum_count_is_shell_size(ora):
    n, box = 16, 50.0
    d, _ = fields(n, box)
    p = ora.RunParams(grid_size=n, box_size=box, which_field=0, n=2, num_values=2, kbinning=0)
    r = ora.ora_run(p, d)
    L = float(np.float32(box))
    for i in range(len(r.k)):
        m = ora.ora_filter(n, 0, r.k[i], 0, 0, 1.0, L)
        assert r.npoly[i] == pytest.approx(float(m.sum()), abs=1e-7)


def test_derived_range_brute_force(ora):
    n, box = 16, 80.0
    L = float(np.float32(box))
    k = 4.3 * 2 * np.pi / L
    mask, kmin, kmax = ora.ora_filter_derived(n, k, 1.0, L)
    idx = np.argwhere(mask)
    m = np.where(idx < n // 2, idx, idx - n).astype(np.float64)
    corners = []
    for sx in (-0.5, 0.5):
        for sy in (-0.5, 0.5):
            for sz in (-0.5, 0.5):
                corners.append((m[:, 0] + sx) ** 2 + (m[:, 1] + sy) ** 2 + (m[:, 2] + sz) ** 2)
    c = np.stack(corners)
    assert kmin == np.sqrt(c.min()) * 2.0 * np.arccos(-1.0) / L
    assert kmax == np.sqrt(c.max()) * 2.0 * np.arccos(-1.0) / L


# ---------------------------------------------------------------- reference
REF_CASES = [
    dict(n=3, equilateral=0, k1=0.2, k2=0.35, num_values=4, kbinning=kb, dcos_theta=0.2,
         use_only_phase=ph, which_field=w)
    for kb in (0, 1, 2, 3) for ph in (0, 1) for w in (0, 2)
] + [
    dict(n=3, equilateral=1, num_values=3, kbinning=kb, dcos_theta=0.1, use_only_phase=0,
         which_field=1)
    for kb in (0, 1, 2, 3)
] + [
    dict(n=2, num_values=2, kbinning=kb, use_only_phase=0, which_field=0) for kb in (0, 2, 3)
]


@pytest.mark.parametrize("case", REF_CASES)
def test_restatement_bit_identical_to_reference(ora, case):
    if not ora.ref_available():
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")
    n, box = 16, 200.0
    d, x = fields(n, box)
    dd, xx = field_args(case["which_field"], d, x)
    p = ora.RunParams(grid_size=n, box_size=box, **case)
    a = ora.ora_run(p, dd, xx)
    b = ora.ref_run(p, dd, xx)
    for f in ("k", "B", "npoly", "kpoly", "kmin", "kmax"):
        np.testing.assert_array_equal(getattr(a, f), getattr(b, f), err_msg=f)


# ---------------------------------------------------------------- golden
def _golden_files():
    return sorted(glob.glob(os.path.join(GOLDEN, "*.json")))


@pytest.mark.parametrize("path", _golden_files(), ids=lambda p: os.path.basename(p))
def test_restatement_matches_golden(ora, path):
    with open(path) as f:
        g = json.load(f)
    n = g["params"]["grid_size"]
    dt = np.float32
    load = lambda name: None if name is None else np.fromfile(os.path.join(GOLDEN, name), dtype=dt).reshape(n, n, n)
    dens, xhii = load(g["dens_file"]), load(g["xhii_file"])
    p = ora.RunParams(**g["params"])
    r = ora.ora_run(p, dens, xhii)
    np.testing.assert_array_equal(r.k, np.array(g["k"]))
    np.testing.assert_array_equal(r.npoly, np.array(g["npoly"]))
    np.testing.assert_array_equal(r.kmin, np.array(g["kmin"]))
    np.testing.assert_array_equal(r.kmax, np.array(g["kmax"]))
    assert rel_err(r.B, np.array(g["B"])).max() <= 1e-12
