"""Build the CUDA library of fastsar_b200 in-tree: fastsar_b200/libffbp_b200.so, for sm_100a only.

    python -m fastsar_b200.build [-v]      # -v: ptxas resource usage (registers, spills, shared memory)

One nvcc invocation over fastsar_b200/csrc/*.cu, -gencode arch=compute_100a,code=sm_100a, linked as a shared
library with the CUDA runtime. The library is rebuilt when a source or the public header is newer than it."""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, 'libffbp_b200.so')
SOURCES = sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cu')))
DEPS = SOURCES + sorted(glob.glob(os.path.join(HERE, 'csrc', '*.h'))) + sorted(glob.glob(os.path.join(HERE, 'csrc', '*.cuh'))) + \
    [os.path.join(ROOT, 'include', 'ffbp_b200.h')]
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']


def nvcc():
    for c in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if c and (os.path.isabs(c) and os.path.exists(c) or not os.path.isabs(c)):
            return c
    return 'nvcc'


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in DEPS)


def build(verbose=False, force=False):
    """Compile the library if it is missing or older than its sources; returns its path."""
    if not force and not stale():
        return LIB
    cmd = [nvcc()] + ARCH + ['-O3', '-lineinfo', '-std=c++17', '--use_fast_math', '-Xcompiler', '-fPIC', '-shared',
                             '-I' + os.path.join(ROOT, 'include'), '-o', LIB + '.tmp'] + SOURCES + ['-lcudart']
    if verbose:
        cmd.insert(1, '-Xptxas=-v')
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('nvcc failed:\n' + ' '.join(cmd) + '\n' + r.stdout + r.stderr)
    if verbose:
        sys.stdout.write(r.stdout + r.stderr)
    os.replace(LIB + '.tmp', LIB)
    return LIB


if __name__ == '__main__':
    build(verbose='-v' in sys.argv, force=True)
    print(LIB)
