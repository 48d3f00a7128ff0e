"""bench.py's reference arm on the CPU: it builds its graph with the host
generator and times the CPU delta-stepping port, loading the oracle library
and none of this package's native code (a reference arm that loaded the
product would not be a reference)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROBE = r"""
import json, runpy, sys
sys.argv = ['bench.py', '--impl', 'reference', '--workload', 'rmat16', '--steps', '3',
            '--warmup', '3']
runpy.run_path('bench.py', run_name='__main__')
maps = open('/proc/self/maps').read()
print(json.dumps({'libadds': 'libadds' in maps, 'liboracle': 'liboracle' in maps}))
"""


def test_reference_arm_loads_only_the_oracle():
    r = subprocess.run([sys.executable, "-c", PROBE], cwd=ROOT, capture_output=True, text=True,
                       timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = [json.loads(x) for x in r.stdout.splitlines() if x.startswith("{")]
    line, maps = lines[0], lines[-1]
    assert line["impl"] == "reference" and line["value"] > 0
    assert line["cpu_baseline"]["kind"] == "port" and "note" in line["cpu_baseline"]
    assert line["e2e"]["h2d_bytes_per_step"] == 0
    assert maps == {"libadds": False, "liboracle": True}
