"""The command-line driver polyspectrum_b200/ps_run on the GPU against the
reference's own executable (oracle/_ref/polyspectrum) on the same ini files
and raw inputs at 32^3: the output files agree line by line - header and the
theta / k columns as text, polygon counts as text (exact integers), B within
the method's tolerance (plain FP64 1e-9 relative, batched FP32 1e-5 relative
plus 1e-6 of the file's max |B|)."""
import os

import numpy as np
import pytest

import oracle
from _driver import make_run, output_file, run_driver

pytestmark = pytest.mark.gpu

CASES = {
    "xhidens_mixed_precision_phase_derived": dict(which=2, gas_dp=0, ion_dp=1, phase=1, n=3, k1=0.11,
                                                  k2=0.16, num_values=6, kbinning=1, box=200.0),
    "dens_double_pk_all_shells": dict(which=0, gas_dp=1, n=2, num_values=2, box=200.0),
    "xhii_float_equilateral_watkinson": dict(which=1, ion_dp=0, n=3, equilateral=1, num_values=4,
                                             kbinning=3, box=200.0),
    "dens_sweep_given_no_counts": dict(which=0, gas_dp=0, n=3, k1=0.1, k2=0.13, num_values=5, kbinning=2,
                                       dcos=0.15, write_np=0, box=200.0),
}


@pytest.fixture(scope="module")
def ref_exe():
    if not oracle.ref_exe_available():
        pytest.fail("oracle/_ref/polyspectrum missing: build it with `make -C oracle ref`")


def read_rows(path):
    with open(path) as f:
        lines = f.read().splitlines()
    return lines[0], [ln.split("\t") for ln in lines[1:]]


@pytest.mark.parametrize("method", ["plain", "batched"])
@pytest.mark.parametrize("name", sorted(CASES))
def test_driver_output_matches_reference(gpu_lib, ref_exe, tmp_path, name, method):
    kw = dict(CASES[name])
    ini = make_run(str(tmp_path), n_grid=32, **kw)
    ref = oracle.run_ref_exe(ini, cwd=str(tmp_path))
    assert ref.returncode == 0, ref.stderr
    fname = os.path.join(str(tmp_path), output_file(ref.stdout))
    ref_head, ref_rows = read_rows(fname)
    os.rename(fname, fname + ".ref")
    ours = run_driver(ini, "--method", method, cwd=str(tmp_path))
    assert ours.returncode == 0, ours.stderr
    head, rows = read_rows(fname)
    assert head == ref_head
    assert len(rows) == len(ref_rows)
    ncols = len(ref_rows[0])
    nkey = 2 if (kw["n"] == 3 and not kw.get("equilateral")) else 1
    has_np = kw.get("write_np", 1) == 1
    bcol = nkey
    Bref = np.array([float(r[bcol]) for r in ref_rows])
    Bgot = np.array([float(r[bcol]) for r in rows])
    scale = np.abs(Bref).max()
    rt, at = (1e-9, 0.0) if method == "plain" else (1e-5, 1e-6)
    for r, g in zip(ref_rows, rows):
        assert len(g) == ncols
        assert g[:nkey] == r[:nkey]
        if has_np:
            assert g[bcol + 1] == r[bcol + 1]
    # %e keeps 7 significant digits: allow one unit in the last printed place
    tol = rt * np.abs(Bref) + at * scale + 1e-6 * np.abs(Bref)
    assert np.all(np.abs(Bgot - Bref) <= tol), (Bgot, Bref)
    # progress lines carry the same k values
    lines = [ln for ln in ours.stdout.splitlines() if ln.startswith(("k = ", "k1 = "))]
    assert len(lines) == len(rows)


def test_driver_exact_sidecar(gpu_lib, ref_exe, tmp_path):
    """ps_run --exact writes <output>.exact: the results at full precision
    ("%.17g"), equal to the C-ABI's batch on the same field and configurations,
    with the DERIVED closing ranges the estimator used; the reference-format
    file beside it rounds the same numbers to "%e"."""
    ps = gpu_lib
    kw = dict(CASES["xhidens_mixed_precision_phase_derived"])
    ini = make_run(str(tmp_path), n_grid=32, **kw)
    ours = run_driver(ini, "--method", "plain", "--exact", cwd=str(tmp_path))
    assert ours.returncode == 0, ours.stderr
    fname = os.path.join(str(tmp_path), output_file(ours.stdout))
    _, rows = read_rows(fname)
    with open(fname + ".exact") as f:
        ex = [[float(x) for x in ln.split("\t")] for ln in f.read().splitlines()[1:]]
    assert len(ex) == len(rows) == kw["num_values"]
    for r, e in zip(rows, ex):
        assert "%e" % e[0] == r[0] and "%e" % e[1] == r[1]
        assert "%e" % e[-2] == r[2] and "%e" % e[-1] == r[3]
    # the same numbers through the C-ABI (double inputs, as ps_run widens mixed precision)
    cfgs, _, _ = ps.read_params_to_kvectors(32, 200.0, 3, k1=kw["k1"], k2=kw["k2"], num_values=kw["num_values"],
                                            kbinningCase=ps.PS_BIN_DERIVED)
    dens = np.fromfile(os.path.join(str(tmp_path), "dens.raw"), dtype=np.float32).astype(np.float64)
    xhii = np.fromfile(os.path.join(str(tmp_path), "xhii.raw"), dtype=np.float64)
    with ps.Context(32, 200.0, methods=ps.PS_FP64_PLAIN) as ctx:
        ctx.get_FT_field(ps.PS_FIELD_XHI_DENS, dens.reshape(32, 32, 32), xhii.reshape(32, 32, 32), use_only_phase=1)
        B, Np, _, out = ctx.batch(cfgs, ps.PS_FP64_PLAIN)
    for i, e in enumerate(ex):
        assert e[-2] == B[i] and e[-1] == Np[i]
        legs = np.array(e[2:-2]).reshape(3, 3)
        np.testing.assert_array_equal(legs[:, 1], list(out[i].kmin)[:3])
        np.testing.assert_array_equal(legs[:, 2], list(out[i].kmax)[:3])


def test_driver_prints_condition_numbers(tmp_path, gpu_lib):
    """Per configuration, ps_run prints the condition number of the value sum
    where the reference prints the imaginary over the real part of its sums
    (polyspectrum.c:142); --no-kappa leaves those lines out."""
    from _driver import make_run, run_driver
    ini = make_run(str(tmp_path), kbinning=1, phase=1)
    out = run_driver(ini, cwd=str(tmp_path), timeout=300)
    assert out.returncode == 0, out.stderr
    lines = [ln for ln in out.stdout.splitlines() if ln.startswith("rank 0: kappa(sumValuesPolygons) = ")]
    assert len(lines) == 4, out.stdout
    for ln in lines:
        assert float(ln.split("=")[1].split()[0]) >= 1.0
    out2 = run_driver(ini, "--no-kappa", cwd=str(tmp_path), timeout=300)
    assert out2.returncode == 0 and "kappa" not in out2.stdout, out2.stdout
