"""CPU checks of the C-ABI boundary: the library loads and exports every
function declared in include/ptbgpu.h; the host mirror's structs match the
header's field lists.  No compute call is made (no GPU here)."""
import ctypes
import re
from pathlib import Path

import pytest

from ptb_b200 import api

HEADER = Path(__file__).resolve().parent.parent / "include" / "ptbgpu.h"


def declared_functions():
    text = HEADER.read_text()
    return sorted(set(re.findall(r"\b(ptbgpu_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    lib = api.load_library()
    names = declared_functions()
    assert len(names) >= 13
    for n in names:
        assert hasattr(lib, n), n
    assert set(names) == set(api.EXPORTED)


def _struct_fields(name):
    text = HEADER.read_text()
    m = re.search(r"typedef struct \{([^{}]*)\}\s*" + name + ";", text)
    assert m, name
    body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
    return re.findall(r"\b(?:int64_t|double)\s+(\w+)\s*;", body)


@pytest.mark.parametrize("cname,pyclass", [("ptbgpu_pur_settings", api._Settings), ("ptbgpu_opts", api._Opts),
                                            ("ptbgpu_stats", api._Stats)])
def test_struct_layouts_match_header(cname, pyclass):
    assert [f for f, _ in pyclass._fields_] == _struct_fields(cname)
    assert ctypes.sizeof(pyclass) == 8 * len(pyclass._fields_)


def test_init_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.PtbGpuError):
        api.Context(0)
