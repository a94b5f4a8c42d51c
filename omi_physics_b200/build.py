"""Build the CUDA library ``_omi_b200.so`` in-tree for sm_100a.

``--fmad=false``: the step must round every multiply and add separately,
as the reference's C accelerators and numpy do; the kernels place their few
deliberate fused operations with explicit ``fma()`` calls.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'csrc', 'omi_b200.cu')
OUT = os.path.join(HERE, '_omi_b200.so')
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


def stale() -> bool:
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    return any(os.path.getmtime(d) > t for d in DEPS)


def build(force: bool = False, verbose: bool = False, extra=()) -> str:
    """Compile the library if any source is newer than it; return its path."""
    if force or stale():
        cmd = [nvcc()] + NVCC_FLAGS + list(extra) + ['-o', OUT, SRC]
        if verbose:
            print(' '.join(cmd))
        subprocess.run(cmd, check=True)
    return OUT


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True,
          extra=['-Xptxas', '-v'] if '--ptxas-v' in sys.argv else [])
