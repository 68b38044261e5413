"""The surrogate-assisted GP's host rules (csrc/sidr_sgp_select.hpp) on the
CPU: ranks with averaged ties, Spearman's rho, the rank-score and
standardised training targets, one-per-key screening in prediction order and
pre-selection by groups -- compiled from the header into a small check
program."""
import os
import subprocess

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
CSRC = os.path.join(REPO, "solver-informed-dispatching-rules_b200", "csrc")


def test_screening_rules(tmp_path):
    exe = tmp_path / "sgp_select_check"
    subprocess.run(["g++", "-std=c++17", "-O2", "-ffp-contract=off", "-Wall", "-I", CSRC,
                    os.path.join(REPO, "tests", "cpp", "sgp_select_check.cpp"), "-o", str(exe)],
                   check=True)
    r = subprocess.run([str(exe)], capture_output=True, text=True)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
