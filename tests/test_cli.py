"""test_dvecchia_batch option parsing (no GPU needed): the reference's flags
and defaults (include/vecchia_helper_data.h:256-739)."""
import json
import os
import subprocess

import pytest

from conftest import ROOT

EXE = os.path.join(ROOT, "blockvecchia_b200", "bin", "test_dvecchia_batch")


@pytest.fixture(scope="module")
def exe(bvlib):
    from blockvecchia_b200 import build
    build.build()
    assert os.path.exists(EXE)
    return EXE


def _opts(exe, *args):
    r = subprocess.run([exe, *args, "--print-opts"], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0, r.stderr
    return json.loads(r.stdout)


def test_defaults(exe):
    o = _opts(exe)
    assert (o["kernel"], o["num_loc"], o["vecchia_cs"], o["vecchia_bc"]) == (1, 2000, 100, 200)
    assert (o["sigma"], o["beta"], o["nu"]) == (1.0, 0.1, 0.5)
    assert (o["sigma_init"], o["beta_init"], o["nu_init"]) == (0.01, 0.01, 0.01)
    assert o["tol"] == 1e-5 and o["maxiter"] == 1000 and o["perf"] == 0 and o["knn"] == 1
    assert (o["lower_bound"], o["upper_bound"]) == (0.01, 3.0)


def test_reference_readme_flags(exe):
    o = _opts(exe, "--vecchia_cs", "300", "--vecchia_bc", "1500", "--kernel",
              "univariate_matern_stationary_no_nugget", "--num_loc", "20000", "--ikernel",
              "1.5:0.1:0.5", "--kernel_init", "0.1:0.1:0.1", "--tol", "4", "--perf", "1",
              "--knn", "1", "--seed", "0")
    assert (o["vecchia_cs"], o["vecchia_bc"], o["num_loc"]) == (300, 1500, 20000)
    assert (o["sigma"], o["beta"], o["nu"]) == (1.5, 0.1, 0.5)
    assert (o["sigma_init"], o["beta_init"], o["nu_init"]) == (0.1, 0.1, 0.1)
    assert o["tol"] == pytest.approx(1e-4) and o["perf"] == 1 and o["maxiter"] == 1


def test_question_mark_keeps_value(exe):
    o = _opts(exe, "--ikernel", "?:0.2:?")
    assert (o["sigma"], o["beta"], o["nu"]) == (1.0, 0.2, 0.5)


@pytest.mark.parametrize("bad", [["--tol", "0"], ["--maxiter", "-3"], ["--upper_bound", "200"],
                                 ["--permutation", "zigzag"], ["--earth", "1"], ["--earth", "--3D", "1"],
                                 ["--kernel", "foo"],
                                 ["--kernel", "univariate_matern_spacetime_stationary", "--t_slots", "3",
                                  "--num_loc", "1000", "--perf", "1"]])
def test_rejected(exe, bad):
    r = subprocess.run([exe, *bad, "--print-opts"], capture_output=True, text=True, timeout=60)
    assert r.returncode != 0 and "error" in r.stderr


def test_spacetime_flags(exe):
    """The space-time kernel's flags (include/vecchia_helper_data.h:505-577):
    seven parameters, six given by --ikernel (aux stays 0), time slots."""
    o = _opts(exe, "--kernel", "univariate_matern_spacetime_stationary", "--ikernel",
              "1.2:0.1:0.5:0.4:0.8:0.6", "--t_slots", "10", "--num_loc", "5000")
    assert o["kernel"] == 4 and o["num_params"] == 7 and o["time_flag"] == 1 and o["t_slots"] == 10
    assert (o["sigma"], o["beta"], o["nu"], o["beta_time"], o["nu_time"], o["sep"]) == \
        (1.2, 0.1, 0.5, 0.4, 0.8, 0.6)
    o = _opts(exe, "--3D", "1")
    assert o["time_flag"] == 1 and o["t_slots"] == 0


@pytest.mark.parametrize("name,code", [("random", 0), ("morton", 1), ("kdtree", 2), ("hilbert", 3),
                                       ("mmd", 4)])
def test_permutation_flag(exe, name, code):
    """--permutation (include/vecchia_helper_data.h:456-476)."""
    o = _opts(exe, "--permutation", name)
    assert o["permutation"] == name and o["ordering"] == code


def test_earth_flag(exe):
    """--earth (include/vecchia_helper_data.h:451-454) sets the great-circle
    metric and does not consume the next argument ("--earth 1" leaves "1" as
    an unrecognised option, as in the reference)."""
    o = _opts(exe, "--earth", "--num_loc", "5000")
    assert o["earth"] == 1 and o["num_loc"] == 5000


def test_precision_flag(exe):
    """--precision mixed keeps FP64 throughout (bv_opts.mixed_fp32 = 0);
    mixed_fp32 forces the FP32 pass."""
    assert (_opts(exe)["precision"], _opts(exe)["mixed_fp32"]) == (0, 0)
    o = _opts(exe, "--precision", "mixed")
    assert (o["precision"], o["mixed_fp32"]) == (1, 0)
    o = _opts(exe, "--precision", "mixed_fp32")
    assert (o["precision"], o["mixed_fp32"]) == (1, 1)
