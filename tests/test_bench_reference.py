"""The bench's reference arm (`bench.py --impl reference`): the timed CPU
restatement of the reference's LSERK4 path prints one JSON line with the
fields the benchmark contract asks of that arm.  CPU only, on a 4^3 sample."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1",
                        "--warmup", "3", "--cells", "4"], capture_output=True, text=True, timeout=600,
                       env=dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0"))
    assert r.returncode == 0, r.stderr[-2000:]
    line = json.loads(r.stdout.strip().splitlines()[-1])
    assert line["impl"] == "reference"
    assert line["metric"] == "DOF-stage-updates/s" and line["unit"] == "DOF-stage/s"
    assert line["value"] > 0 and line["higher_is_better"] is True
    assert line["warmup"] >= 3 and line["steps"] == 1
    cb = line["cpu_baseline"]
    assert cb["kind"] == "port" and cb["cores"] >= 1 and cb["value"] == line["value"]
    e2e = line["e2e"]
    assert e2e["value"] == line["value"] and e2e["h2d_bytes_per_step"] == 0 and e2e["d2h_bytes_per_step"] == 0
    assert line["config"]["cells"] == "4^3" and line["config"]["n_dof"] == 6 * 4 ** 3 * 35 * 6
    assert line["finite"] is True


def test_reference_arm_loads_no_product_code():
    """The reference arm builds its mesh, materials and initial field with the
    oracle alone: the product's native library is never mapped."""
    code = (
        "import sys, types; sys.argv = ['bench.py', '--impl', 'reference', '--steps', '1', '--warmup', '1', "
        "'--cells', '3']; sys.path.insert(0, %r); import bench; bench.main(); "
        "maps = open('/proc/self/maps').read(); "
        "assert 'librapidfem_b200' not in maps, 'product library mapped'; "
        "assert 'libdgtd_oracle' in maps; "
        "assert not any(m.startswith('rapidfem_b200') for m in sys.modules), 'product module imported'"
    ) % ROOT
    r = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, RANK="0", WORLD_SIZE="1", LOCAL_RANK="0"))
    assert r.returncode == 0, r.stderr[-2000:]


def test_reference_arm_other_ranks_do_nothing():
    r = subprocess.run([sys.executable, os.path.join(ROOT, "bench.py"), "--impl", "reference", "--steps", "1"],
                       capture_output=True, text=True, timeout=300,
                       env=dict(os.environ, RANK="1", WORLD_SIZE="2", LOCAL_RANK="1"))
    assert r.returncode == 0 and r.stdout.strip() == ""
