"""Build the sorter's shared library in-tree: ``livespikesorter_b200/liblss_b200.so``.

Every CUDA source is compiled for sm_100a only (``-gencode
arch=compute_100a,code=sm_100a``); nvcc cross-compiles without a GPU.
Objects go to ``_build/`` next to the sources; a source is recompiled when it or
any header is newer than its object.

    python -m livespikesorter_b200.build [--verbose-ptxas]
"""
from __future__ import annotations

import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / 'csrc'
INCLUDE = PKG.parent / 'include'
BUILD = PKG / '_build'
LIB = PKG / 'liblss_b200.so'
NVCC = os.environ.get('NVCC', '/usr/local/cuda/bin/nvcc')
ARCH = ['-gencode', 'arch=compute_100a,code=sm_100a']
FLAGS = ['-O3', '-lineinfo', '-std=c++17', '-Xcompiler', '-fPIC', '--expt-relaxed-constexpr',
         '-I', str(CSRC), '-I', str(INCLUDE)]


def _sources():
    return sorted(list(CSRC.glob('*.cu')) + list(CSRC.glob('*.cpp')))


def _headers():
    return list(CSRC.glob('*.h')) + list(CSRC.glob('*.cuh')) + list(INCLUDE.glob('*.h'))


def _compile(src: Path, ptxas_verbose: bool) -> Path:
    obj = BUILD / (src.name + '.o')
    newest_dep = max([src.stat().st_mtime] + [h.stat().st_mtime for h in _headers()])
    if obj.exists() and obj.stat().st_mtime >= newest_dep:
        return obj
    cmd = [NVCC, *ARCH, *FLAGS, '-c', str(src), '-o', str(obj)]
    if ptxas_verbose and src.suffix == '.cu':
        cmd += ['-Xptxas', '-v']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'nvcc failed for {src.name}:\n{r.stdout}\n{r.stderr}')
    if ptxas_verbose:
        sys.stdout.write(r.stderr)
    return obj


def build(ptxas_verbose: bool = False) -> Path:
    BUILD.mkdir(exist_ok=True)
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as ex:
        objs = list(ex.map(lambda s: _compile(s, ptxas_verbose), _sources()))
    if LIB.exists() and LIB.stat().st_mtime >= max(o.stat().st_mtime for o in objs):
        return LIB
    tmp = LIB.with_suffix('.so.tmp')
    # --no-undefined: a symbol missing from the sources fails the build, not the first dlopen
    cmd = [NVCC, *ARCH, '-shared', '-Xlinker', '--no-undefined', '-o', str(tmp), *map(str, objs), '-lcudart_static',
           '-lrt', '-ldl', '-lpthread']
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f'link failed:\n{r.stdout}\n{r.stderr}')
    os.replace(tmp, LIB)
    return LIB


if __name__ == '__main__':
    print(build(ptxas_verbose='--verbose-ptxas' in sys.argv))
