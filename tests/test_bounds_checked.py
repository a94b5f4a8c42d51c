"""The bounds-checked debug library (``_omi_b200_checked.so``, no GPU): it is
built from the same source with ``-DOMI_BOUNDS_CHECK``, exports every symbol
the header declares, says which build it is, is the one the package loads
under ``OMI_B200_CHECKED=1``, and its failure code maps to its own Python
exception. Its device checks run on the GPU in ``test_gpu_zbounds_checked.py``.
"""
import ctypes
import os
import subprocess
import sys

import pytest

from omi_physics_b200 import _lib, build
from test_abi import declared_functions

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope='module')
def libraries():
    return ctypes.CDLL(build.build()), ctypes.CDLL(build.build(checked=True))


def test_each_build_says_which_it_is(libraries):
    shipped, checked = libraries
    assert shipped.omi_bounds_checked() == 0
    assert checked.omi_bounds_checked() == 1


def test_checked_build_exports_every_declared_symbol(libraries):
    _, checked = libraries
    missing = [name for name in declared_functions() if not hasattr(checked, name)]
    assert not missing


def test_environment_selects_the_checked_build(libraries):
    code = ('from omi_physics_b200 import _lib; lib = _lib.load_library(); '
            'print(_lib.LIB_PATH == _lib.LIB_PATH_CHECKED, lib.omi_bounds_checked())')
    for value, want in (('1', 'True 1'), ('0', 'False 0'), ('', 'False 0')):
        env = dict(os.environ, OMI_B200_CHECKED=value, PYTHONPATH=ROOT)
        out = subprocess.run([sys.executable, '-c', code], env=env, cwd=ROOT, capture_output=True, text=True,
                             check=True).stdout.split()
        assert ' '.join(out[-2:]) == want, (value, out)


def test_a_failed_check_raises_its_own_exception():
    class FakeLib:
        @staticmethod
        def omi_last_error(h):
            return b'1 device index check(s) failed, the first at narrowphase pair body (index 99)'

    ctx = _lib.Context.__new__(_lib.Context)
    ctx.lib, ctx.h = FakeLib(), None
    with pytest.raises(_lib.BoundsError) as err:
        ctx.check(_lib.OMI_E_BOUNDS, 'omi_step')
    assert err.value.code == -8 and 'narrowphase pair body' in str(err.value)
    assert issubclass(_lib.BoundsError, _lib.OmiError)
