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
