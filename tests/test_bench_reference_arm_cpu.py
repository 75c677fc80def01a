"""The reference arm of bench.py (`--impl reference`) on the host cores.

It times the reference's own CPU engine (oracle/_ref/rtm, built from the
reference's sources) migrating whole shots of the config-3 survey, one per step,
and prints one JSON line with the same metric, unit and config as the library's
arm.  These tests run it for one short step (nt cut to 200 so the test stays
quick) and check the line's keys, that ranks other than 0 print nothing and exit
0, and that the arm never imports the engine package or maps librtm_b200.so, so
the driver's record of loaded libraries shows the reference alone.
"""
import json
import os
import subprocess
import sys

import pytest

import oracle

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_RTM = oracle.ref_binary("rtm")


def _run(env_extra, extra_args=()):
    env = dict(os.environ)
    env.update(env_extra)
    return subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                           "--warmup", "0", "--nt", "200", *extra_args], capture_output=True, text=True, env=env,
                          timeout=600, cwd=ROOT)


@pytest.mark.skipif(REF_RTM is None, reason="reference binaries not built into oracle/_ref")
def test_reference_arm_prints_the_contract_line():
    r = _run({"RANK": "0"})
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "shots/s" and line["unit"] == "shots/s" and line["higher_is_better"] is True
    assert line["value"] > 0 and line["steps"] == 1 and line["warmup"] == 0
    assert line["config"]["workload"].startswith("config3")
    cb = line["cpu_baseline"]
    assert cb["kind"] == "reference" and cb["cores"] >= 1 and cb["sample"] and cb["value"] == line["value"]
    assert "x86-64-v3" in cb["sample"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["unit"] == line["unit"]
    assert e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0


def test_reference_arm_other_ranks_do_no_work():
    r = _run({"RANK": "1", "WORLD_SIZE": "2", "LOCAL_RANK": "1"})
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == ""


@pytest.mark.skipif(REF_RTM is None, reason="reference binaries not built into oracle/_ref")
def test_reference_arm_never_loads_the_engine():
    code = ("import sys, json; sys.argv=['bench.py']; sys.path.insert(0, %r); import bench; "
            "bench.main(['--impl', 'reference', '--steps', '1', '--warmup', '0', '--nt', '120']); "
            "maps = open('/proc/self/maps').read(); "
            "print(json.dumps({'pkg': any(m.startswith('rtm_b200') for m in sys.modules), "
            "'so': 'librtm_b200' in maps}))") % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, cwd=ROOT, timeout=600,
                       env=dict(os.environ, RANK="0"))
    assert r.returncode == 0, r.stderr[-2000:]
    seen = json.loads(r.stdout.strip().splitlines()[-1])
    assert seen == {"pkg": False, "so": False}
