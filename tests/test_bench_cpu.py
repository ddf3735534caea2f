"""bench.py's command line on CPU: the contract the benchmark driver relies on (flags, the
workload table) holds without a GPU; the runs themselves are GPU work."""
import importlib.util
import re
import subprocess
import sys
from pathlib import Path

ROOT = Path(__file__).resolve().parents[1]


def _bench_module():
    spec = importlib.util.spec_from_file_location("bench_cli", ROOT / "bench.py")
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)  # defines functions only; main() runs under __main__
    return mod


def test_help_lists_the_driver_flags():
    out = subprocess.run([sys.executable, str(ROOT / "bench.py"), "--help"], capture_output=True, text=True,
                         timeout=120)
    assert out.returncode == 0, out.stderr
    for flag in ("--gpus", "--steps", "--warmup", "--impl", "--workload"):
        assert flag in out.stdout, flag


def test_every_workload_choice_has_a_runner():
    mod = _bench_module()
    text = (ROOT / "bench.py").read_text()
    block = text[text.index('"--workload"'):]
    choices = re.findall(r'"([a-z0-9-]+)"', block[block.index("choices=["):block.index("]")])
    assert choices[0] == "mixed-n1048576"  # the default: the headline workload
    assert set(choices[1:]) == set(mod.OTHER_WORKLOADS)
