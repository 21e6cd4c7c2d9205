"""Build recipe for the sm_100a shared library ``rqutils_b200/lib/libsqd_b200.so``.

The library is a plain C-ABI shared object (see ``include/sqd_b200.h``) compiled with nvcc for
``sm_100a`` only; the CUDA runtime is linked statically so the object does not depend on the
runtime that PyTorch ships.  Objects are rebuilt when a source or header is newer.
"""
import os
import shutil
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, 'csrc')
LIBDIR = os.path.join(HERE, 'lib')
BUILDDIR = os.path.join(ROOT, '_build')
LIBNAME = 'libsqd_b200.so'
LIBPATH = os.path.join(LIBDIR, LIBNAME)

ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
NVCC_FLAGS = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '-Xcompiler', '-Wall',
              '--expt-relaxed-constexpr', '-I', os.path.join(ROOT, 'include')]


def nvcc_path():
    for cand in (os.environ.get('NVCC'), shutil.which('nvcc'), '/usr/local/cuda/bin/nvcc'):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError('nvcc not found')


def _sources():
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith('.cu'))


def _headers():
    hdrs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.cuh', '.h'))]
    hdrs.append(os.path.join(ROOT, 'include', 'sqd_b200.h'))
    return hdrs


def _newer(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False, jobs=None):
    """Compile every .cu under csrc/ and link the shared library.  Returns its path."""
    nvcc = nvcc_path()
    os.makedirs(BUILDDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    hdrs = _headers()
    objs = []
    todo = []
    for src in _sources():
        obj = os.path.join(BUILDDIR, os.path.basename(src)[:-3] + '.o')
        objs.append(obj)
        if _newer(obj, [src] + hdrs) or ptxas_info:
            cmd = [nvcc, *ARCH, *NVCC_FLAGS, '-c', src, '-o', obj]
            if ptxas_info:
                cmd.insert(1, '-Xptxas=-v')
            todo.append(cmd)

    def run(cmd):
        if verbose:
            print(' '.join(cmd), flush=True)
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f'nvcc failed:\n{" ".join(cmd)}\n{res.stdout}\n{res.stderr}')
        return res.stdout + res.stderr

    with ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 1)) as ex:
        logs = list(ex.map(run, todo))
    if ptxas_info:
        for log in logs:
            print(log)
    if todo or _newer(LIBPATH, objs):
        tmp = LIBPATH + '.tmp'
        run([nvcc, *ARCH, '-shared', '-o', tmp, *objs, '-lcudart_static', '-ldl', '-lrt',
             '-lpthread'])
        os.replace(tmp, LIBPATH)
    return LIBPATH


if __name__ == '__main__':
    print(build(verbose='-v' in sys.argv, ptxas_info='--ptxas' in sys.argv))
