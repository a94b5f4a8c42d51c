"""Build the CUDA library ``_omi_b200.so`` in-tree for sm_100a.

``--fmad=false``: the step must round every multiply and add separately,
as the reference's C accelerators and numpy do; the kernels place their few
deliberate fused operations with explicit ``fma()`` calls.

``--checked`` builds the bounds-checked debug library ``_omi_b200_checked.so``
instead (``-DOMI_BOUNDS_CHECK``: device index checks that skip a bad access
and make the step report OMI_E_BOUNDS); ``OMI_B200_CHECKED=1`` loads it.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'csrc', 'omi_b200.cu')
OUT = os.path.join(HERE, '_omi_b200.so')
OUT_CHECKED = os.path.join(HERE, '_omi_b200_checked.so')
DEPS = [os.path.join(HERE, 'csrc', f) for f in os.listdir(os.path.join(HERE, 'csrc'))]
DEPS.append(os.path.join(os.path.dirname(HERE), 'include', 'omi_b200.h'))

NVCC_FLAGS = [
    '-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo',
    '--fmad=false', '-Xcompiler', '-fPIC', '-shared', '-Xptxas', '-O3',
]


def nvcc() -> str:
    for cand in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if cand and (os.path.sep not in cand or os.path.exists(cand)):
            return cand
    return 'nvcc'


def stale(out: str = OUT) -> bool:
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra=(), checked: bool = False) -> str:
    """Compile the library (the bounds-checked one with ``checked``) if any
    source is newer than it; return its path."""
    out = OUT_CHECKED if checked else OUT
    if force or stale(out):
        cmd = [nvcc()] + NVCC_FLAGS + (['-DOMI_BOUNDS_CHECK'] if checked else []) + list(extra) + ['-o', out, SRC]
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
    return out


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True,
          extra=['-Xptxas', '-v'] if '--ptxas-v' in sys.argv else [], checked='--checked' in sys.argv)
