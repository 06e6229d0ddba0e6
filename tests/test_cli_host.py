"""Command-line handling of the drop-in tools that needs no GPU: the return
codes and usage text of bin/ancandidates mirror the reference's ANcandidates
(ANcandidates/ANcandidates.cpp:165-233)."""
import subprocess
from pathlib import Path

import pytest

import oracle

ROOT = Path(__file__).resolve().parent.parent
EXE = ROOT / "coding_reliability_b200" / "bin" / "ancandidates"


def run(*args):
    return subprocess.run([str(EXE)] + list(args), capture_output=True, text=True, timeout=60)


def test_help_returns_255_with_the_reference_usage():
    r = run("-h")
    assert r.returncode == 255
    usage = r.stdout.splitlines()
    assert usage[0] == "USAGE: /ancandidates -a|--Amin -A|--Amax -d|--dMin -D|--dMax"
    if oracle.ref_ancandidates_available():
        ref = subprocess.run([str(oracle.REF_OUT / "ref_ancandidates"), "--help"], capture_output=True, text=True)
        assert ref.returncode == 255
        ref_lines = ref.stdout.replace("ref_ancandidates", "ancandidates").splitlines()
        assert usage[:len(ref_lines)] == ref_lines


@pytest.mark.parametrize("args", [[], ["-a", "2", "-A", "4"], ["-d", "0", "-D", "3", "-a", "1", "-A", "2"]])
def test_missing_width_returns_100(args):
    assert run(*args).returncode == 100


@pytest.mark.parametrize("flag,code", [("-a", 1), ("--Amax", 2), ("-d", 3), ("--Dmax", 4)])
def test_flag_without_value(flag, code):
    r = run(flag)
    assert r.returncode == code and "requires an additional number" in r.stderr


def test_empty_range_is_refused():
    assert run("-a", "5", "-A", "4", "-d", "2", "-D", "3").returncode == 5
