"""Build libuppe_b200.so in-tree with nvcc for sm_100a (no GPU needed)."""
import concurrent.futures
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
BUILD = os.path.join(HERE, '_build')
LIB = os.path.join(HERE, 'libuppe_b200.so')
SOURCES = ['uppe3d.cu', 'uppe1d.cu', 'uppe1d_f32.cu', 'uppe1d_f64.cu', 'uppe1d_noalloc.cu', 'uppe1d_cl_f32.cu',
           'uppe1d_cl_f64.cu', 'uppe_probe.cu']
HEADERS = ['common.cuh', 'uppe1d_kernel.cuh', 'uppe1d_cluster.cuh']
NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '-std=c++17',
              '-Xcompiler', '-fPIC', '-Xcompiler', '-O2']


def _nvcc():
    for c in (os.environ.get('CUDA_HOME', ''), '/usr/local/cuda'):
        p = os.path.join(c, 'bin', 'nvcc')
        if c and os.path.exists(p):
            return p
    return 'nvcc'


def _deps():
    files = [os.path.join(CSRC, f) for f in SOURCES + HEADERS]
    files.append(os.path.join(os.path.dirname(HERE), 'include', 'uppe_b200.h'))
    files.append(os.path.abspath(__file__))
    return [f for f in files if os.path.exists(f)]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(f) <= t for f in _deps())


def _includes(path, seen=None):
    """The source file and the local headers it includes, recursively."""
    seen = set() if seen is None else seen
    if path in seen or not os.path.exists(path):
        return seen
    seen.add(path)
    with open(path) as f:
        for line in f:
            line = line.strip()
            if line.startswith('#include "'):
                name = line.split('"')[1]
                for d in (os.path.dirname(path), os.path.join(os.path.dirname(HERE), 'include')):
                    q = os.path.normpath(os.path.join(d, name))
                    if os.path.exists(q):
                        _includes(q, seen)
                        break
    return seen


def _object_current(src, obj):
    """An object is current when it is newer than its source, the headers that
    source includes and this build script."""
    if not os.path.exists(obj):
        return False
    t = os.path.getmtime(obj)
    deps = _includes(os.path.join(CSRC, src)) | {os.path.abspath(__file__)}
    return all(os.path.getmtime(f) <= t for f in deps)


def build(force=False, verbose=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(BUILD, exist_ok=True)
    nvcc = _nvcc()
    srcs = [s for s in SOURCES if os.path.exists(os.path.join(CSRC, s))]

    def compile_one(src):
        obj = os.path.join(BUILD, src.replace('.cu', '.o'))
        if not force and _object_current(src, obj):
            return obj
        cmd = [nvcc] + NVCC_FLAGS + ['-c', os.path.join(CSRC, src), '-o', obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'nvcc failed for {src}:\n{r.stdout}\n{r.stderr}')
        if verbose:
            print(r.stderr, file=sys.stderr)
        return obj

    with concurrent.futures.ThreadPoolExecutor(max_workers=len(srcs)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB + '.tmp'
    cmd = [nvcc, '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', '-o', tmp] + objs + ['-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stdout}\n{r.stderr}')
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
