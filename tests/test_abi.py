"""The C-ABI library builds, loads and exports every symbol of include/lss.h;
host-side argument checks that need no GPU."""
import ctypes
import re
import subprocess

import pytest

from conftest import ROOT


@pytest.fixture(scope='module')
def lib():
    from livespikesorter_b200 import build, _lib
    build.build()
    return _lib.load()


def declared_symbols():
    text = (ROOT / 'include' / 'lss.h').read_text()
    text = re.sub(r'/\*.*?\*/', '', text, flags=re.S)
    return sorted(set(re.findall(r'\b(lss_[a-z_]+)\s*\(', text)))


def test_header_declares_the_binding_exports():
    from livespikesorter_b200 import _lib
    assert declared_symbols() == sorted(_lib.EXPORTS)


def test_library_exports_every_declared_symbol(lib):
    from livespikesorter_b200 import _lib
    out = subprocess.run(['nm', '-D', '--defined-only', str(_lib.LIB_PATH)], capture_output=True, text=True).stdout
    exported = set(re.findall(r'\b(lss_[a-z_]+)\b', out))
    for sym in declared_symbols():
        assert sym in exported, sym
        assert hasattr(lib, sym)


def test_library_is_sm100a_only(lib):
    from livespikesorter_b200 import _lib
    out = subprocess.run(['/usr/local/cuda/bin/cuobjdump', '--list-elf', str(_lib.LIB_PATH)],
                         capture_output=True, text=True).stdout
    assert 'sm_100a' in out
    assert not re.search(r'sm_(?!100a)\d+', out)


def test_create_rejects_bad_config_without_gpu(lib):
    from livespikesorter_b200._lib import LssConfig, LssTensors, LSS_ERR_ARG
    h = ctypes.c_void_p()
    cfg = LssConfig(n_chan=4, n_chan_bin=4, n_templates=2, n_pcs=2, nt=20, n_nearest=0, batch_size=100,
                    nt0min=5, th_learned=8.0, max_rounds=100, max_spikes=10, do_car=1)
    rc = lib.lss_create(cfg, LssTensors(), ctypes.byref(h))
    assert rc == LSS_ERR_ARG
    assert b'odd' in lib.lss_last_error(None)
    cfg.nt = 21
    cfg.n_pcs = 9
    assert lib.lss_create(cfg, LssTensors(), ctypes.byref(h)) == LSS_ERR_ARG
    cfg.n_pcs = 2
    assert lib.lss_create(cfg, LssTensors(), ctypes.byref(h)) == LSS_ERR_ARG  # missing tensors
    assert b'required' in lib.lss_last_error(None)


def test_create_from_missing_dir_is_io_error(lib, tmp_path):
    from livespikesorter_b200._lib import LSS_ERR_IO
    h = ctypes.c_void_p()
    assert lib.lss_create_from_dir(str(tmp_path / 'nope').encode(), None, ctypes.byref(h)) == LSS_ERR_IO
    assert b'Wall3.npy' in lib.lss_last_error(None)


def test_python_api_fails_loudly_without_library(monkeypatch, tmp_path):
    from livespikesorter_b200 import _lib
    monkeypatch.setattr(_lib, '_lib', None)
    monkeypatch.setattr(_lib, 'LIB_PATH', tmp_path / 'missing.so')
    with pytest.raises(ImportError, match='no CPU fallback'):
        _lib.load()


def test_plain_c_program_links_and_calls_the_abi(lib, tmp_path):
    """include/lss.h is C99 and liblss_b200.so links into a C program."""
    exe = tmp_path / 'c_caller'
    libdir = ROOT / 'livespikesorter_b200'
    subprocess.run(['gcc', '-std=c99', '-Wall', '-Wextra', '-Werror', '-pedantic', '-I', str(ROOT / 'include'),
                    str(ROOT / 'tests' / 'c' / 'c_caller.c'), '-o', str(exe), '-L', str(libdir), '-llss_b200',
                    f'-Wl,-rpath,{libdir}'], check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    assert out == '1100,3,12.5,0\n1250,0,0.25,0\ncreate=1 handle=null error=yes\n'
