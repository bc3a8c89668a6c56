"""Build the engine in-tree (sm_100a only).

    python -m hfpx3d_b200.build          # -> hfpx3d_b200/libhfpx_engine.so
                                         #    hfpx3d_b200/libhfpx_host.so
                                         #    hfpx3d_b200/bin/hfpx_main

libhfpx_engine.so is the CUDA engine behind the C-ABI (include/hfpx_engine.h);
libhfpx_host.so the C++ host layer over it (host/hfpx.hpp); hfpx_main the
config.toml driver.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
HOST = os.path.join(HERE, 'host')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
OUT = os.path.join(HERE, 'libhfpx_engine.so')
HOST_LIB = os.path.join(HERE, 'libhfpx_host.so')
LAPACKE_LIB = os.path.join(HERE, 'libhfpx_lapacke.so')
MAIN = os.path.join(HERE, 'bin', 'hfpx_main')
SOURCES = ['engine.cu', 'assembly.cu', 'lu.cu', 'solve.cu', 'gemm_tc.cu', 'precond.cu', 'gnn.cu', 'vc.cu', 'batch.cu',
           'coarse.cu', 'cf.cu']
CUDA = os.environ.get('CUDA_HOME', '/usr/local/cuda')
NVCC = os.path.join(CUDA, 'bin', 'nvcc')
CXX = os.environ.get('CXX', 'g++')
FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-O3', '-std=c++17',
         '-Xcompiler', '-fPIC', '-shared', '--expt-relaxed-constexpr', '-I' + INCLUDE]
LIBS = ['-L' + os.path.join(CUDA, 'lib64'), '-lcublas', '-lcusolver', '-Xlinker', '-rpath=' + os.path.join(CUDA, 'lib64')]
# --exclude-libs: a toolchain that links its C++ runtime statically must not
# re-export it from these libraries into the programs that load them
HOST_FLAGS = ['-O2', '-std=c++17', '-Wall', '-I' + INCLUDE, '-I' + HOST, '-Wl,--exclude-libs,ALL']


def _stale(out, deps):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(d) > t for d in deps)


def needs_build():
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)]
    deps.append(os.path.join(INCLUDE, 'hfpx_engine.h'))
    return _stale(OUT, deps)


def _run(cmd, verbose):
    if verbose:
        print(' '.join(cmd))
    subprocess.run(cmd, check=True)


def build_host(force=False, verbose=False):
    """C++ host layer and driver, linked against libhfpx_engine.so (rpath
    $ORIGIN, so the tree can move as a whole)."""
    deps = [os.path.join(HOST, f) for f in os.listdir(HOST)] + [OUT, os.path.join(INCLUDE, 'hfpx_engine.h')]
    if force or _stale(HOST_LIB, deps):
        _run([CXX] + HOST_FLAGS + ['-fPIC', '-shared', os.path.join(HOST, 'hfpx_host.cpp'), '-o', HOST_LIB,
                                   '-L' + HERE, '-lhfpx_engine', '-Wl,-rpath,$ORIGIN'], verbose)
    if force or _stale(MAIN, deps + [HOST_LIB]):
        os.makedirs(os.path.dirname(MAIN), exist_ok=True)
        _run([CXX] + HOST_FLAGS + [os.path.join(HOST, 'hfpx_main.cpp'), '-o', MAIN, '-L' + HERE, '-lhfpx_host',
                                   '-lhfpx_engine', '-Wl,-rpath,$ORIGIN/..'], verbose)
    if force or _stale(LAPACKE_LIB, deps):
        _run([CXX] + HOST_FLAGS + ['-fPIC', '-shared', os.path.join(HOST, 'lapacke_shim.cpp'), '-o', LAPACKE_LIB,
                                   '-L' + HERE, '-lhfpx_engine', '-Wl,-rpath,$ORIGIN'], verbose)
    return MAIN


def build(force=False, verbose=False):
    if force or needs_build():
        _run([NVCC] + FLAGS + [os.path.join(CSRC, s) for s in SOURCES] + ['-o', OUT] + LIBS, verbose)
    build_host(force, verbose)
    return OUT


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose=True))
