"""Build liboi_b200.so in-tree: every CUDA source under csrc/, compiled for sm_100a only.

    python -m opticalimaging_b200.build [--force]

The library lands in opticalimaging_b200/_lib/ so it travels with the source tree.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
INCLUDE = os.path.join(os.path.dirname(HERE), 'include')
LIBDIR = os.path.join(HERE, '_lib')
LIB = os.path.join(LIBDIR, 'liboi_b200.so')
NVCC_FLAGS = ['-gencode', 'arch=compute_100a,code=sm_100a', '-O3', '-lineinfo', '-std=c++17',
              '-Xcompiler', '-fPIC', '-Xcompiler', '-fvisibility=hidden', '-I', INCLUDE]


def sources():
    return sorted(glob.glob(os.path.join(CSRC, '*.cu')))


def deps():
    return sources() + glob.glob(os.path.join(CSRC, '*.cuh')) + glob.glob(os.path.join(INCLUDE, '*.h'))


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    return any(os.path.getmtime(p) > t for p in deps())


def build(force=False, verbose=False):
    """Compile the sources to objects (in parallel) and link the shared library.  Returns its path."""
    if not force and not stale():
        return LIB
    nvcc = os.environ.get('NVCC', 'nvcc')
    objdir = os.path.join(LIBDIR, 'obj')
    os.makedirs(objdir, exist_ok=True)
    procs = []
    objs = []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + '.o')
        objs.append(obj)
        cmd = [nvcc, *NVCC_FLAGS, '-c', src, '-o', obj]
        if verbose:
            print(' '.join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode(errors='replace')))
    if failed:
        raise RuntimeError('nvcc failed:\n' + '\n'.join(f'--- {s}\n{o}' for s, o in failed))
    tmp = LIB + '.tmp'
    cmd = [nvcc, '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', *objs, '-o', tmp, '-lcudart']
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)
    if r.returncode != 0:
        raise RuntimeError('link failed:\n' + r.stdout.decode(errors='replace'))
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
