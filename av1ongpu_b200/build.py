"""Builds the libraries in-tree.

    python -m av1ongpu_b200.build        (or import and call build())

libav1b.so - the decoder: the sm_100a kernels, the host engine and the C ABI
(csrc/). nvcc compiles the .cu files for sm_100a only (no PTX for other
targets), the host compiler the .cpp files.
libav1synth.so - the seeded workload generator (synth/), host code only, kept
apart so that a process that only needs the workload maps no decoder code.

Both land next to this file, where the Python package and the tests load
them. Objects live in av1ongpu_b200/_build/ and are rebuilt when a source or
header is newer.
"""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, 'csrc')
SYNTH_SRC = os.path.join(HERE, 'synth')
OUT = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libav1b.so')
SYNTH_LIB = os.path.join(HERE, 'libav1synth.so')
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
CXX = '/usr/bin/g++'
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVFLAGS = ARCH + ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler',
                  '-fvisibility=hidden', '-diag-suppress', '68', '-I', SRC]
CXXFLAGS = ['-O2', '-std=c++17', '-fPIC', '-fvisibility=hidden', '-I', SRC,
            '-I', '/usr/local/cuda/include']


def _headers():
    roots = [SRC, SYNTH_SRC, os.path.join(os.path.dirname(HERE), 'include')]
    out = []
    for r in roots:
        for dirpath, _, files in os.walk(r):
            out += [os.path.join(dirpath, f) for f in files if f.endswith(('.h', '.hpp', '.cuh'))]
    return out


def _stale(obj, src, deps_mtime):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return os.path.getmtime(src) > t or deps_mtime > t


def _compile(src, obj):
    if src.endswith('.cu'):
        cmd = [NVCC] + NVFLAGS + ['-c', src, '-o', obj]
    else:
        cmd = [CXX] + CXXFLAGS + ['-c', src, '-o', obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError('compile failed: %s\n%s%s' % (' '.join(cmd), r.stdout, r.stderr))
    return obj


def _build_lib(src_dir, lib, link, verbose):
    """Compiles what changed under src_dir and links `lib`."""
    os.makedirs(OUT, exist_ok=True)
    sources = sorted(os.path.join(src_dir, f) for f in os.listdir(src_dir)
                     if f.endswith(('.cu', '.cpp')))
    deps = max(os.path.getmtime(h) for h in _headers())
    jobs = []
    objs = []
    for s in sources:
        obj = os.path.join(OUT, os.path.basename(s) + '.o')
        objs.append(obj)
        if _stale(obj, s, deps):
            jobs.append((s, obj))
    if jobs:
        with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, len(jobs))) as ex:
            for obj in ex.map(lambda j: _compile(*j), jobs):
                if verbose:
                    print('built', os.path.basename(obj))
    if jobs or not os.path.exists(lib) or max(os.path.getmtime(o) for o in objs) > os.path.getmtime(lib):
        cmd = link(objs)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError('link failed: %s\n%s%s' % (' '.join(cmd), r.stdout, r.stderr))
    return lib


def build(verbose=False):
    """Compiles what changed and links libav1b.so and libav1synth.so. Returns
    the decoder library's path."""
    _build_lib(SYNTH_SRC, SYNTH_LIB, lambda objs: [CXX, '-shared', '-o', SYNTH_LIB] + objs, verbose)
    return _build_lib(SRC, LIB, lambda objs: [NVCC] + ARCH + ['-shared', '-o', LIB] + objs +
                      ['-lcudart_static', '-lpthread', '-ldl', '-lrt'], verbose)


if __name__ == '__main__':
    print(build(verbose='-v' in sys.argv))
