"""The command-line driver polyspectrum_b200/ps_run without a GPU: ini parsing,
configuration lists, output file names and the reference's error exits,
checked against the reference's own executable (oracle/_ref/polyspectrum,
serial, run on the same ini files at 16^3).  ps_run --dry-run stops before it
reads the inputs or touches a device."""
import os

import pytest

import oracle
from _driver import dry_run_configs, make_run, output_file, run_driver


@pytest.fixture(scope="module")
def tools():
    from polyspectrum_b200 import build
    build.build(quiet=True)
    if not oracle.ref_exe_available() and oracle.reference_checkout() is not None:
        oracle.build_oracle(ref=True)
    if not oracle.ref_exe_available():
        pytest.skip("oracle/_ref not built (needs the reference checkout at build time)")


CASES = {
    "sweep_default": dict(n=3, k1=0.2, k2=0.3, num_values=4),
    "sweep_one_theta": dict(n=3, k1=0.2, k2=0.3, num_values=1, theta=0.7),
    "sweep_derived": dict(n=3, k1=0.25, k2=0.3, num_values=5, kbinning=1),
    "sweep_given": dict(n=3, k1=0.2, k2=0.35, num_values=3, kbinning=2, dcos=0.2),
    "sweep_watkinson": dict(n=3, k1=0.2, k2=0.35, num_values=3, kbinning=3, dcos=0.2),
    "equilateral": dict(n=3, equilateral=1, num_values=5),
    "equilateral_given": dict(n=3, equilateral=1, num_values=3, kbinning=2),
    "pk_all_shells": dict(n=2, num_values=3),
    "pk_no_counts": dict(n=2, num_values=3, write_np=0),
}


def text_columns(path):
    with open(path) as f:
        lines = f.read().splitlines()
    return lines[0], [ln.split("\t") for ln in lines[1:]]


@pytest.mark.parametrize("name", sorted(CASES))
def test_dry_run_matches_reference(tools, tmp_path, name):
    kw = CASES[name]
    ini = make_run(str(tmp_path), **kw)
    ref = oracle.run_ref_exe(ini, cwd=str(tmp_path))
    assert ref.returncode == 0, ref.stderr
    ours = run_driver(ini, "--dry-run", cwd=str(tmp_path))
    assert ours.returncode == 0, ours.stderr
    assert ours.stdout.splitlines()[0] == ref.stdout.splitlines()[0]  # kbinningCase = %d
    fname = output_file(ref.stdout)
    assert output_file(ours.stdout) == fname
    _, rows = text_columns(os.path.join(str(tmp_path), fname))
    cfg = dry_run_configs(ours.stdout)
    assert len(cfg) == len(rows)
    for (theta, k), row in zip(cfg, rows):
        if kw["n"] == 3 and not kw.get("equilateral"):
            assert row[0] == "%e" % theta and row[1] == "%e" % k
        else:
            assert row[0] == "%e" % k


def _both(tmp_path, args=(), **kw):
    ini = make_run(str(tmp_path), **kw)
    ref = oracle.run_ref_exe(ini, cwd=str(tmp_path))
    ours = run_driver(ini, *args, cwd=str(tmp_path))
    return ref, ours


@pytest.mark.parametrize("drop", ["Y", "gridsize", "kbinningCase", "write_numpolygons"])
def test_missing_key_exits_like_reference(tools, tmp_path, drop):
    ref, ours = _both(tmp_path, ("--dry-run",), drop_keys=(drop,))
    assert ref.returncode != 0 and ours.returncode != 0
    assert ours.stderr.strip() == ref.stderr.strip()
    assert "FATAL:  Could not get %s" % drop in ours.stderr


def test_missing_use_only_phase_is_optional(tools, tmp_path):
    ref, ours = _both(tmp_path, ("--dry-run",), drop_keys=("useOnlyPhase",))
    assert ref.returncode == 0 and ours.returncode == 0


def test_missing_output_dir(tools, tmp_path):
    ref, ours = _both(tmp_path, ("--dry-run",), out_dir="no_such_dir")
    assert ref.returncode != 0 and ours.returncode != 0
    assert ours.stderr.strip() == ref.stderr.strip() == "Directory for output does not exist!"


def test_unknown_field(tools, tmp_path):
    ref, ours = _both(tmp_path, which="RHO")
    assert ref.returncode != 0 and ours.returncode != 0
    assert ours.stderr.strip() == ref.stderr.strip()
    assert ours.stdout.splitlines()[-1].startswith("Option: RHO")


def test_n_above_three(tools, tmp_path):
    ref, ours = _both(tmp_path, ("--dry-run",), n=4)
    assert ref.returncode != 0 and ours.returncode != 0
    assert ours.stdout.strip() == ref.stdout.strip() == "Not implemented yet"


def test_malformed_line(tools, tmp_path):
    ref, ours = _both(tmp_path, ("--dry-run",), extra_lines=("this line has no separator",))
    assert ref.returncode != 0 and ours.returncode != 0
    assert ours.stderr == ref.stderr


def test_usage(tools):
    from _driver import PS_RUN
    import subprocess
    r = subprocess.run([PS_RUN], capture_output=True, text=True)
    assert r.returncode != 0 and "USAGE" in r.stdout
