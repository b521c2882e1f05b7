"""CPU checks of the top-level scripts: every global name a function of
bench.py or __graft_entry__.py reads is defined (their GPU paths cannot run
here), and the benchmark's reference arm prints its JSON line."""
import builtins
import json
import subprocess
import sys
import symtable
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


def _undefined_globals(path: Path):
    top = symtable.symtable(path.read_text(), str(path), "exec")
    defined = {s.get_name() for s in top.get_symbols() if s.is_assigned() or s.is_imported()}
    defined |= set(dir(builtins)) | {"__file__", "__name__"}
    bad = []

    def walk(t):
        for s in t.get_symbols():
            if t.get_type() == "function" and s.is_global() and s.is_referenced() and s.get_name() not in defined:
                bad.append(f"{t.get_name()}: {s.get_name()}")
        for c in t.get_children():
            walk(c)

    walk(top)
    return bad


@pytest.mark.parametrize("name", ["bench.py", "__graft_entry__.py"])
def test_scripts_reference_only_defined_globals(name):
    assert _undefined_globals(ROOT / name) == []


def test_bench_reference_arm_prints_one_json_line():
    r = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--impl", "reference", "--config", "1", "--steps", "1",
                        "--warmup", "0", "--cpu-pairs", "20000"], capture_output=True, text=True, timeout=600,
                       cwd=ROOT)
    assert r.returncode == 0, r.stderr
    lines = [ln for ln in r.stdout.splitlines() if ln.strip()]
    assert len(lines) == 1
    out = json.loads(lines[0])
    assert out["impl"] == "reference" and out["unit"] == "nets/s" and out["value"] > 0
    assert out["cpu_baseline"]["kind"] == "port"
    assert out["e2e"]["h2d_bytes_per_step"] == 0 and out["e2e"]["d2h_bytes_per_step"] == 0
