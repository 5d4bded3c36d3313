"""Build libmbpt_b200.so in-tree with nvcc for sm_100a.

    python -m mbptcode_b200.build

The library is a plain shared object with a C ABI (include/mbpt_b200.h); the
Python package loads it with ctypes, so no torch headers are involved.
"""
from __future__ import annotations

import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, 'csrc')
ROOT = os.path.dirname(HERE)
LIB = os.path.join(HERE, 'libmbpt_b200.so')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
SOURCES = ['gemm_host.cu', 'kernels.cu', 'aux_kernels.cu', 'capi.cu', 'qp.cu', 'mlp.cu',
           'noalloc.cu', 'contour.cu', 'ozaki.cu']
# files whose arithmetic must round as written (no FMA contraction)
NO_FMA = {'qp.cu'}


def nvcc():
    for c in (os.environ.get('NVCC'), '/usr/local/cuda/bin/nvcc', 'nvcc'):
        if c and (os.path.sep not in c or os.path.exists(c)):
            return c
    return 'nvcc'


def build(verbose=False, jobs=None):
    objdir = os.path.join(HERE, '_build')
    os.makedirs(objdir, exist_ok=True)
    base = [nvcc(), *ARCH, '-O3', '-std=c++17', '-lineinfo', '-Xcompiler', '-fPIC',
            '-I', os.path.join(ROOT, 'include'), '--expt-relaxed-constexpr']
    objs, procs = [], []
    newest_hdr = max(os.path.getmtime(os.path.join(CSRC, f)) for f in os.listdir(CSRC))
    newest_hdr = max(newest_hdr, os.path.getmtime(os.path.join(ROOT, 'include', 'mbpt_b200.h')))
    for src in SOURCES:
        obj = os.path.join(objdir, src.replace('.cu', '.o'))
        objs.append(obj)
        if os.path.exists(obj) and os.path.getmtime(obj) >= newest_hdr:
            continue
        cmd = base + (['-fmad=false'] if src in NO_FMA else []) + \
            ['-c', os.path.join(CSRC, src), '-o', obj]
        if verbose:
            print(' '.join(cmd))
        procs.append((src, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((src, out.decode()))
        elif verbose and out:
            print(out.decode())
    if failed:
        for src, out in failed:
            sys.stderr.write(f'--- {src}\n{out}\n')
        raise RuntimeError('nvcc failed for ' + ', '.join(s for s, _ in failed))
    link = [nvcc(), *ARCH, '-shared', '-o', LIB, *objs, '-lcublas', '-lcusolver']
    if verbose:
        print(' '.join(link))
    subprocess.run(link, check=True)
    return LIB


if __name__ == '__main__':
    print(build(verbose='-v' in sys.argv))
