"""Build the engine's CUDA shared library in-tree (sm_100a only).

    python -m hfpx3d_b200.build          # -> hfpx3d_b200/libhfpx_engine.so
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, 'libhfpx_engine.so')
SOURCES = ['engine.cu', 'assembly.cu', 'lu.cu']
CUDA = os.environ.get('CUDA_HOME', '/usr/local/cuda')
NVCC = os.path.join(CUDA, 'bin', 'nvcc')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3', '-std=c++17',
         '-Xcompiler', '-fPIC', '-shared', '--expt-relaxed-constexpr',
         '-I' + os.path.join(os.path.dirname(HERE), 'include')]
LIBS = ['-L' + os.path.join(CUDA, 'lib64'), '-lcublas', '-Xlinker', '-rpath=' + os.path.join(CUDA, 'lib64')]


def needs_build():
    if not os.path.exists(OUT):
        return True
    t = os.path.getmtime(OUT)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(os.path.dirname(HERE), 'include', 'hfpx_engine.h'))
    return any(os.path.getmtime(d) > t for d in deps)


def build(force=False, verbose=False):
    if not force and not needs_build():
        return OUT
    cmd = [NVCC] + FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ['-o', OUT] + LIBS
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
