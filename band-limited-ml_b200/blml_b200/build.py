"""Build libblml_b200.so in-tree with nvcc for sm_100a (python -m blml_b200.build)."""
import os
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
REPO = os.path.dirname(ROOT)
CSRC = os.path.join(ROOT, 'csrc')
INCLUDE = os.path.join(REPO, 'include')
LIB = os.path.join(PKG, 'libblml_b200.so')
SOURCES = ['capi.cu', 'matvec.cu', 'fft_matvec.cu', 'tc_matvec.cu', 'solver_ops.cu', 'pairs.cu', 'batched.cu', 'batch_runner.cu', 'unet.cu',
           'points.cu', 'predict.cu']
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
FLAGS = ['-O3', '-std=c++17', '-gencode', 'arch=compute_100a,code=sm_100a', '-lineinfo', '-Xcompiler', '-fPIC',
         '-Xcompiler', '-O3', '--expt-relaxed-constexpr', '-I', INCLUDE, '-I', CSRC]


def stale():
    if not os.path.exists(LIB):
        return True
    t = os.path.getmtime(LIB)
    deps = [os.path.join(CSRC, f) for f in os.listdir(CSRC)] + [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return any(os.path.getmtime(p) > t for p in deps)


def build(force=False, verbose=False, jobs=None):
    """Compile every source to an object and link the shared library (skipped when it is newer than its sources)."""
    if not force and not stale():
        return LIB
    objdir = os.path.join(ROOT, '_build')
    os.makedirs(objdir, exist_ok=True)
    from concurrent.futures import ThreadPoolExecutor

    def compile_one(src):
        obj = os.path.join(objdir, src.replace('.cu', '.o'))
        cmd = [NVCC] + FLAGS + ['-c', os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f'nvcc failed on {src}:\n{r.stderr}')
        if verbose and r.stderr:
            print(r.stderr, flush=True)
        return obj

    with ThreadPoolExecutor(jobs or len(SOURCES)) as ex:
        objs = list(ex.map(compile_one, SOURCES))
    tmp = LIB + '.tmp'
    cmd = [NVCC, '-shared', '-gencode', 'arch=compute_100a,code=sm_100a', '-o', tmp] + objs + ['-lcudart']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stderr}')
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build(force='--force' in sys.argv, verbose='-v' in sys.argv))
