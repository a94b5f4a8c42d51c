"""bench.py's reference arm on CPU: one JSON line with the contract's keys
(the GPU arm is exercised on the B200)."""
import json
import os
import subprocess
import sys

import pytest

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


def test_clock_sampler_reads_nvml_and_summarises(monkeypatch):
    """The sampler against a fake NVML module: median SM clock, max clock and
    the slowdown reasons seen while it ran (only read-only queries are made)."""
    import types
    sys.path.insert(0, ROOT)
    import bench
    calls = []
    clocks = iter([1965, 1965, 1800, 1965] + [1965] * 1000)
    fake = types.SimpleNamespace(
        NVML_CLOCK_SM=1, nvmlClocksEventReasonHwSlowdown=0x8, nvmlClocksEventReasonHwThermalSlowdown=0x40,
        nvmlClocksEventReasonSwThermalSlowdown=0x20, nvmlClocksEventReasonSwPowerCap=0x4,
        nvmlInit=lambda: calls.append('init'), nvmlShutdown=lambda: calls.append('shutdown'),
        nvmlDeviceGetHandleByPciBusId=lambda bus: 'h',
        nvmlDeviceGetHandleByIndex=lambda i: 'h',
        nvmlDeviceGetClockInfo=lambda h, c: next(clocks),
        nvmlDeviceGetMaxClockInfo=lambda h, c: 1965,
        nvmlDeviceGetCurrentClocksEventReasons=lambda h: 0x4)
    monkeypatch.setitem(sys.modules, 'pynvml', fake)
    with bench.ClockSampler(0) as clk:
        import time
        time.sleep(0.03)
    s = clk.summary()
    assert calls[0] == 'init' and calls[-1] == 'shutdown'
    assert s['samples'] >= 3 and s['sm_max_mhz'] == 1965 and s['sm_mhz'] == 1965
    assert s['reasons'] == ['sw_power_cap']


@pytest.mark.gpu
@pytest.mark.parametrize('args', [
    ['--worlds', '24', '--steps', '3', '--warmup', '3', '--preroll', '10', '--no-extras'],
    ['--workload', 'pyramid', '--config-steps', '6', '--no-extras'],
])
def test_bench_runs_end_to_end_and_prints_its_line(args):
    """bench.py itself, small: it exits 0 and prints one JSON line with the
    contract's keys (a crash here would cost the measured run)."""
    import json
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    res = subprocess.run([sys.executable, os.path.join(root, 'bench.py')] + args, capture_output=True,
                         text=True, timeout=900, cwd=root)
    assert res.returncode == 0, res.stderr[-2000:]
    line = json.loads(res.stdout.strip().splitlines()[-1])
    for key in ('metric', 'value', 'unit', 'n_gpus', 'steps', 'warmup', 'ms_per_step', 'higher_is_better',
                'scaling', 'dtype', 'config', 'e2e', 'roofline', 'clocks', 'gpu_launches', 'tuning'):
        assert key in line, key
    assert line['value'] > 0 and line['gpu_launches'] > 0
