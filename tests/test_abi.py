"""The C-ABI library: every symbol include/omi_b200.h declares is exported and
bound, and the Python binding's struct mirrors match the header (no GPU)."""
import ctypes
import os
import re

import pytest

from omi_physics_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, 'include', 'omi_b200.h')


def declared_functions():
    text = open(HEADER).read()
    return sorted(set(re.findall(r'^\s*(?:const\s+)?\w+\s*\*?\s*(omi_\w+)\s*\(', text, re.M)))


@pytest.fixture(scope='module')
def library():
    build.build()
    return ctypes.CDLL(_lib.LIB_PATH)


def test_header_and_binding_agree():
    decl = declared_functions()
    assert len(decl) >= 30
    assert set(decl) == set(_lib.PROTOTYPES)


def test_library_exports_every_declared_symbol(library):
    missing = [name for name in declared_functions() if not hasattr(library, name)]
    assert not missing


def test_struct_mirrors_match_header_fields():
    text = open(HEADER).read()
    body = text[text.index('typedef struct OmiScene {'):text.index('} OmiScene;')]
    names = re.findall(r'\*?(\w+)\s*[,;]', re.sub(r'/\*.*?\*/', '', body, flags=re.S))
    names = [n for n in names if n not in ('int32_t', 'double', 'uint8_t')]
    assert names == [f for f, _ in _lib.OmiScene._fields_]
    caps = text[text.index('typedef struct OmiSlotCaps {'):text.index('} OmiSlotCaps;')]
    cap_names = re.findall(r'(\w+)[,;]', caps.split('{', 1)[1])
    assert cap_names == [f for f, _ in _lib.OmiSlotCaps._fields_]


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, 'LIB_PATH', str(tmp_path / 'absent.so'))
    monkeypatch.setattr(_lib, '_LIB', None)
    with pytest.raises(_lib.OmiError):
        _lib.load_library()
