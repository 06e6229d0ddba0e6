"""The drop-in command lines on the GPU against the reference's own outputs:
bin/codrel against the stdout of the reference's codrel (CPU paths, recorded in
tests/golden/ref_runs.json) and bin/codrel_supera against the output files of
the reference's super-A tool (its GPU path, tests/golden/supera_ref.json).
Run-time figures and device descriptions differ by nature and are dropped
before comparing; everything else must be identical."""
import json
import re
import subprocess
from pathlib import Path

import pytest

pytestmark = pytest.mark.gpu

ROOT = Path(__file__).resolve().parent.parent
BIN = ROOT / "coding_reliability_b200" / "bin"
GOLD = ROOT / "tests" / "golden"
RUNTIME = re.compile(r'^\d+,"(Total|Kernel) Runtime",')


def normalise_codrel(text):
    return [l for l in text.splitlines() if not RUNTIME.match(l)]


REF_RUNS = json.loads((GOLD / "ref_runs.json").read_text())


@pytest.mark.parametrize("case", REF_RUNS, ids=lambda c: " ".join(c["args"]))
def test_codrel_stdout_matches_reference(case, tmp_path):
    r = subprocess.run([str(BIN / "codrel")] + case["args"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    assert normalise_codrel(r.stdout) == normalise_codrel(case["stdout"])


def normalise_supera(text):
    """Rows of a super-A results file without the time columns (t_kernel, t)
    and without the device lines and the total-time line."""
    out = []
    for line in text.splitlines():
        if not line or line.startswith('"'):
            continue
        f = [x.strip() for x in line.split(",")]
        if f[0] == "id" or not f[0].isdigit():
            out.append(line)
            continue
        cnts = int(f[7])
        t = 8 + 2 * cnts
        out.append(",".join(f[:t] + f[t + 2:]))
    return out


SUPERA = json.loads((GOLD / "supera_ref.json").read_text()) if (GOLD / "supera_ref.json").exists() else None


@pytest.mark.skipif(SUPERA is None, reason="supera_ref.json not generated")
@pytest.mark.parametrize("idx", range(len(SUPERA["cases"])) if SUPERA else [])
def test_codrel_supera_file_matches_reference(idx, tmp_path):
    case = SUPERA["cases"][idx]
    (tmp_path / "cand.csv").write_text(SUPERA["candidates_file"])
    r = subprocess.run([str(BIN / "codrel_supera")] + case["args"], capture_output=True, text=True, cwd=tmp_path,
                       timeout=600)
    assert r.returncode == 0, r.stderr
    out = tmp_path / case["file"]
    assert out.exists(), sorted(p.name for p in tmp_path.iterdir())
    got, want = normalise_supera(out.read_text()), normalise_supera(case["content"])
    assert len(got) == len(want) and got == want
