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
