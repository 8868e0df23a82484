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


@pytest.mark.parametrize("what", ["short", "missing"])
def test_input_file_errors(tools, tmp_path, what):
    """A short or missing input grid ends the run with an error before any
    device is touched (ps_run checks each file's size and first value, then
    the library streams it)."""
    ini = make_run(str(tmp_path), n_grid=16, which=2, gas_dp=0, ion_dp=1)
    path = tmp_path / "xhii.raw"
    if what == "short":
        data = path.read_bytes()
        path.write_bytes(data[: len(data) // 2])
    else:
        path.unlink()
    ours = run_driver(ini, cwd=str(tmp_path))
    assert ours.returncode != 0
    msg = ("xhii.raw holds 2048 of the 4096 values of the grid" if what == "short"
           else "cannot open input file xhii.raw")
    assert msg in ours.stderr


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


# ---------------------------------------------------------------- ini-file generator
CREATE_INI = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "polyspectrum_b200",
                          "ps_create_ini")
INI_ARGS = ["64", "100.3", "0", "1", "dens.raw", "xhii.raw", "0.7", "0.0456", "0.27", "0.73", "0.82", "0.24",
            "XHI_DENS", "PHASE", "3", "0", "0.25", "0.3", "5", "0.1", "1.0", "DERIVED", "0.2", "out", "run", "1"]


def _ini_args(phase):
    """The generator's positional arguments (useOnlyPhase in slot 14 when given)."""
    a = list(INI_ARGS)
    if phase is None:
        a.remove("PHASE")
    else:
        a[a.index("PHASE")] = str(phase)
    return a


@pytest.fixture(scope="module")
def ini_tools():
    from polyspectrum_b200 import build
    build.build_create_ini()
    ref_dir = os.path.join(os.path.dirname(oracle.__file__), "_ref")
    if not os.path.exists(os.path.join(ref_dir, "create_inifile_phase")) and oracle.reference_checkout() is not None:
        oracle.build_oracle(ref=True)
    return ref_dir


@pytest.mark.parametrize("phase", [None, 0, 1], ids=["no_phase_key", "phase0", "phase1"])
def test_create_ini_matches_reference_generator(ini_tools, tmp_path, phase):
    """Byte-for-byte the file of the reference's generator (main.c without the
    useOnlyPhase argument, main_withOptionPhase.c with it)."""
    import subprocess
    ref_exe = os.path.join(ini_tools, "create_inifile" if phase is None else "create_inifile_phase")
    if not os.path.exists(ref_exe):
        pytest.skip("reference generators not built (needs the reference checkout at build time)")
    args = _ini_args(phase)
    ours = subprocess.run([CREATE_INI, str(tmp_path / "ours.ini"), *args], capture_output=True, text=True)
    ref = subprocess.run([ref_exe, str(tmp_path / "ref.ini"), *args], capture_output=True, text=True)
    assert ours.returncode == 0 and ref.returncode == 0, (ours.stderr, ref.stderr)
    assert (tmp_path / "ours.ini").read_bytes() == (tmp_path / "ref.ini").read_bytes()


def test_create_ini_wrong_argument_count(ini_tools, tmp_path):
    """A wrong argument count is an error exit with the usage (the reference
    writes through an uninitialised file name there)."""
    import subprocess
    r = subprocess.run([CREATE_INI, str(tmp_path / "x.ini"), "64"], capture_output=True, text=True)
    assert r.returncode == 1 and "usage" in r.stderr
    assert not (tmp_path / "x.ini").exists()


def test_generated_ini_runs_like_reference(tools, ini_tools, tmp_path):
    """A generated ini file drives ps_run --dry-run to the configurations and
    output file name of the reference executable on the same file."""
    import subprocess
    make_run(str(tmp_path), n_grid=16, box=100.0)  # the inputs dens.raw / xhii.raw
    args = _ini_args(1)
    args[0], args[1] = "16", "100.0"
    ini = str(tmp_path / "gen.ini")
    assert subprocess.run([CREATE_INI, ini, *args]).returncode == 0
    ref = oracle.run_ref_exe(ini, cwd=str(tmp_path))
    assert ref.returncode == 0, ref.stderr
    ours = run_driver(ini, "--dry-run", cwd=str(tmp_path))
    assert ours.returncode == 0, ours.stderr
    fname = output_file(ref.stdout)
    assert output_file(ours.stdout) == fname
    _, rows = text_columns(os.path.join(str(tmp_path), fname))
    cfg = dry_run_configs(ours.stdout)
    assert len(cfg) == len(rows) == 5
    for (theta, k), row in zip(cfg, rows):
        assert row[0] == "%e" % theta and row[1] == "%e" % k
