"""Register and stack use of the hot kernels (no GPU: nvcc's resource report).

The contact sweep keeps a run's bodies, rows and impulses in registers; if
the compiler stops inlining its body into ``k_iterate``, the arena it takes
by reference goes to the stack and the sweep slows by ~10%. This pins the
resource use of the step's hot kernels and of the capsule-triangle kernel:
no stack frame and no spills, registers within the budget that keeps their
occupancy.
"""
import os
import re
import shutil
import subprocess

import pytest

from omi_physics_b200 import build

LIMITS = {            # kernel name fragment -> register ceiling
    'k_iterate': 224,
    'k_wsweep': 224,
    'k_prep': 128,
    'k_finalize': 64,
    'k_pair_count': 64,
    'k_pair_emit': 64,
    'k_sort': 64,
    'k_refit': 96,
    'k_integrate_forces': 64,
    'k_capsule_triangles': 128,
    'k_joints': 128,
}


@pytest.fixture(scope='module')
def report(tmp_path_factory):
    nvcc = build.nvcc()
    if not shutil.which(nvcc) and not os.path.exists(nvcc):
        pytest.skip('nvcc not available')
    out = str(tmp_path_factory.mktemp('res') / 'probe.so')
    cmd = [nvcc] + build.NVCC_FLAGS + ['-Xptxas', '-v', '-o', out, build.SRC]
    res = subprocess.run(cmd, capture_output=True, text=True, check=True)
    kernels, cur = {}, None
    for line in (res.stdout + res.stderr).splitlines():
        m = re.search(r'Function properties for (\S+)', line)
        if m:
            cur = m.group(1)
            continue
        if cur is None:
            continue
        m = re.search(r'(\d+) bytes stack frame, (\d+) bytes spill stores, (\d+) bytes spill loads', line)
        if m:
            kernels.setdefault(cur, {}).update(stack=int(m.group(1)), spill=int(m.group(2)) + int(m.group(3)))
        m = re.search(r'Used (\d+) registers', line)
        if m:
            kernels.setdefault(cur, {})['regs'] = int(m.group(1))
    return kernels


@pytest.mark.parametrize('name', sorted(LIMITS))
def test_hot_kernels_keep_their_resources(report, name):
    found = {k: v for k, v in report.items() if name in k}
    assert found, name
    for k, v in found.items():
        assert v.get('stack', 0) == 0 and v.get('spill', 0) == 0, (k, v)
        assert v['regs'] <= LIMITS[name], (k, v)
