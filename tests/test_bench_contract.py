"""bench.py's reference arm on CPU: one JSON line with the contract's keys
(the GPU arm is exercised on the B200)."""
import json
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_reference_arm_json_line():
    out = subprocess.run([sys.executable, os.path.join(ROOT, 'bench.py'), '--impl', 'reference', '--worlds', '4',
                          '--preroll', '5', '--cpu-sample-s', '1', '--steps', '2', '--warmup', '1'],
                         capture_output=True, text=True, timeout=300, cwd=ROOT)
    assert out.returncode == 0, out.stderr[-2000:]
    lines = [l for l in out.stdout.splitlines() if l.strip().startswith('{')]
    assert len(lines) == 1
    d = json.loads(lines[0])
    assert d['impl'] == 'reference'
    if 'unavailable' in d:                       # the reference was not built here
        assert not os.path.isdir(os.path.join(ROOT, 'oracle', '_ref', 'omi_physics'))
        return
    for k in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'higher_is_better', 'scaling', 'dtype',
              'data', 'config', 'cpu_baseline', 'e2e'):
        assert k in d, k
    assert d['value'] > 0 and d['higher_is_better'] is True and d['scaling'] == 'weak'
    assert d['config']['workload'] == 'serving-mix'
    cb = d['cpu_baseline']
    assert cb['kind'] == 'reference' and cb['cores'] >= 1 and cb['value'] == d['value']
    assert set(d['e2e']) >= {'value', 'unit', 'h2d_bytes_per_step', 'd2h_bytes_per_step'}
