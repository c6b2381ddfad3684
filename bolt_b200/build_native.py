"""Build the CUDA shared library of bolt_b200 (sm_100a) in-tree.

    python -m bolt_b200.build_native          # -> bolt_b200/_native/libbolt_b200.so

The FP64 kernels are compiled with -fmad=false so that their arithmetic
follows the reference's operation order; the FP32 kernels and the FP64
kernel of the fast FP64 form use FMA and approximate division (FP32) or
Newton-refined reciprocals (FP64).  The library links the CUDA runtime statically and
loads cuTensorMapEncodeTiled through the runtime's driver entry point.
"""

import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
OUT_DIR = os.path.join(HERE, '_native')
LIB = os.path.join(OUT_DIR, 'libbolt_b200.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
COMMON = ['-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
          '-I', os.path.join(HERE, '..', 'include')]
UNITS = [
    ('kernels_f64.cu', ['-fmad=false']),
    ('kernels_f32.cu', ['-prec-div=false', '-prec-sqrt=false', '-ftz=true']),
    ('kernels_f64pair.cu', []),
    ('bolt_capi.cu', []),
    ('bolt_noalloc.cu', []),
    ('bolt_batch.cu', ['-prec-div=false', '-prec-sqrt=false', '-ftz=true']),
    ('bolt_adjoint.cu', []),
    ('poisson.cu', ['-fmad=false']),
]


def nvcc():
    exe = shutil.which('nvcc') or '/usr/local/cuda/bin/nvcc'
    if not os.path.exists(exe):
        raise RuntimeError('nvcc not found')
    return exe


def sources():
    return [os.path.join(CSRC, f) for f in os.listdir(CSRC)
            if f.endswith(('.cu', '.cuh', '.h'))] + \
        [os.path.join(HERE, '..', 'include', 'bolt_b200.h')]


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(s) <= t for s in sources())


def build(force=False, verbose=False, ptxas_v=False):
    if not force and up_to_date():
        return LIB
    os.makedirs(OUT_DIR, exist_ok=True)
    objs, cmds = [], []
    for src, extra in UNITS:
        obj = os.path.join(OUT_DIR, src.replace('.cu', '.o'))
        cmd = [nvcc()] + ARCH + COMMON + extra + ['-c', os.path.join(CSRC, src), '-o', obj]
        if ptxas_v:
            cmd += ['-Xptxas', '-v']
        if verbose:
            print(' '.join(cmd))
        cmds.append(cmd)
        objs.append(obj)
    # the units are independent: compile them side by side
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=max(1, min(len(cmds), os.cpu_count() or 1))) as ex:
        for res in list(ex.map(lambda c: subprocess.run(c, capture_output=True, text=True), cmds)):
            sys.stdout.write(res.stdout)
            sys.stderr.write(res.stderr)
            if res.returncode != 0:
                raise subprocess.CalledProcessError(res.returncode, res.args)
    cmd = [nvcc()] + ARCH + ['-shared', '-o', LIB] + objs + ['-lcufft']
    subprocess.run(cmd, check=True)
    for o in objs:
        os.remove(o)
    return LIB


if __name__ == '__main__':
    build(force='--force' in sys.argv, verbose=True, ptxas_v='--ptxas-v' in sys.argv)
    print(LIB)
