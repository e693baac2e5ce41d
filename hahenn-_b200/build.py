"""Build libsuiri_cuda.so in-tree with nvcc for sm_100a (B200).

    python hahenn-_b200/build.py          # or build() from Python

Objects go to hahenn-_b200/_build/, the library to hahenn-_b200/libsuiri_cuda.so. The files whose results
are compared bit for bit (binning, obstacle geometry and face fractions, the cell pass and the pressure
solve, the emitters, the distance queries and the surface mesh) are built without FMA contraction (-fmad=false), so that their
float64 geometry and float32 pressure arithmetic round exactly as written; the grid-to-particle pass and the
ripple layer, held to tolerances, let the compiler contract.
"""
import concurrent.futures as cf
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT = os.path.join(HERE, 'libsuiri_cuda.so')
BUILD = os.path.join(HERE, '_build')
NVCC = os.environ.get('NVCC', 'nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC,-O3', '--expt-relaxed-constexpr']
SOURCES = ['bin.cu', 'grid.cu', 'sor.cu', 'g2p.cu', 'ripple.cu', 'mesh.cu', 'engine.cu', 'scene.cpp', 'server.cpp',
           'capi.cpp']
CONTRACTED = {'g2p.cu', 'ripple.cu'}      # tolerance-checked results: FMA contraction allowed


def _compile(src, verbose):
    obj = os.path.join(BUILD, os.path.splitext(src)[0] + '.o')
    path = os.path.join(CSRC, src)
    deps = [path] + [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith(('.h', '.cuh'))]
    deps.append(os.path.join(os.path.dirname(HERE), 'include', 'suiri.h'))
    if os.path.exists(obj) and os.path.getmtime(obj) >= max(os.path.getmtime(d) for d in deps):
        return obj
    fmad = '-fmad=true' if src in CONTRACTED else '-fmad=false'
    cmd = [NVCC, *ARCH, *FLAGS, fmad, '-c', path, '-o', obj]
    if verbose:
        print(' '.join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc failed on {src}:\n{r.stdout}\n{r.stderr}')
    return obj


def build(verbose=False, force=False):
    """Compile every CUDA/C++ source of the library and link libsuiri_cuda.so. Returns its path."""
    os.makedirs(BUILD, exist_ok=True)
    if force:
        for f in os.listdir(BUILD):
            os.remove(os.path.join(BUILD, f))
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 2)) as ex:
        objs = list(ex.map(lambda s: _compile(s, verbose), SOURCES))
    if os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(o) for o in objs):
        return OUT
    cmd = [NVCC, *ARCH, '-shared', '-cudart=static', '-o', OUT, *objs]
    if verbose:
        print(' '.join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stdout}\n{r.stderr}')
    return OUT


if __name__ == '__main__':
    print(build(verbose=True, force='--force' in sys.argv))
