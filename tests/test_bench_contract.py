"""The two bench arms print lines the driver can pair: the same metric
string, unit and direction, the requested steps and warm-up, and a reference
arm that builds its box without loading the product library."""
import json
import subprocess
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent.parent

PROBE = r"""
import json, sys, types
sys.path.insert(0, {root!r})
import bench
args = types.SimpleNamespace(workload="lj_solvent_4096", seed=2024, steps=2, warmup=1)
bench.run_reference_arm(args, 1, 0)
maps = open("/proc/self/maps").read()
print(json.dumps({{"product_loaded": "liblima_b200.so" in maps,
                   "libs": sorted({{l.split()[-1] for l in maps.splitlines() if l.endswith(".so")
                                    and "/oracle/" in l}})}}))
"""


def test_reference_arm_loads_no_product_library_and_matches_the_metric():
    r = subprocess.run([sys.executable, "-c", PROBE.format(root=str(ROOT))], cwd=ROOT, capture_output=True,
                       text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(l) for l in r.stdout.splitlines() if l.startswith("{")]
    assert len(lines) == 2
    line, probe = lines
    sys.path.insert(0, str(ROOT))
    import bench
    assert line["metric"] == bench.metric_name("lj_solvent_4096")
    assert line["unit"] == "ns/day" and line["higher_is_better"] is True
    assert line["steps"] == 2 and line["warmup"] == 1
    assert not probe["product_loaded"], probe
    assert all("/oracle/" in p for p in probe["libs"])


def test_oracle_packer_is_bit_identical_to_the_product_packer():
    from quantom_b200 import systems as S
    a = S.make_system("tiny_chains", seed=3)
    b = S.make_system("tiny_chains", seed=3, packer_lib=ROOT / "oracle" / "liblima_inputs.so")
    for f in ("solvents", "compounds", "states"):
        assert np.array_equal(getattr(a, f).view(np.uint8), getattr(b, f).view(np.uint8)), f
