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


C_CALLER = r"""
#include <stdio.h>
#include <string.h>
#include "ptbgpu.h"

int main(void) {
    ptbgpu_pur_settings s;
    ptbgpu_opts o;
    ptbgpu_stats st;
    int32_t tiles[4 * 64];
    int64_t nt = 0, info[4];
    ptbgpu_ctx* c = NULL;
    int rc;
    ptbgpu_default_settings(&s);
    ptbgpu_default_opts(&o);
    memset(&st, 0, sizeof st);
    if (s.type != PTBGPU_TYPE_DIAG || s.cycles != 40 || s.chempot_cycles != 60 || s.chempot_guess != -1.5)
        return 2;
    if (o.precision != PTBGPU_PREC_MIXED) return 3;
    rc = ptbgpu_oz_tiles(256, 8, 64, 0, 0, 0, 0, tiles, 64, &nt, info);
    if (rc != PTBGPU_OK || nt <= 0) return 4;
    if (ptbgpu_oz_tiles(0, 8, 64, 0, 0, 0, 0, tiles, 64, &nt, info) != PTBGPU_EINVAL) return 5;
    rc = ptbgpu_init(0, &c);
    printf("init %d tiles %lld\n", rc, (long long)nt);
    if (rc == PTBGPU_OK) ptbgpu_finalize(c);
    return 0;
}
"""


def test_header_compiles_as_c99_and_links(tmp_path):
    """A C caller (what the Fortran ISO_C_BINDING shim binds to) compiles against
    the header with -std=c99 -pedantic -Werror, links libptbgpu and makes the
    host-only calls; without a GPU, ptbgpu_init returns a status instead of
    failing the process."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("no C compiler")
    lib = api.library_path()
    src = tmp_path / "caller.c"
    src.write_text(C_CALLER)
    exe = tmp_path / "caller"
    cmd = [gcc, "-std=c99", "-pedantic", "-Wall", "-Wextra", "-Werror", f"-I{HEADER.parent}", str(src),
           f"-L{lib.parent}", "-l:" + lib.name, f"-Wl,-rpath,{lib.parent}", "-Wl,--allow-shlib-undefined",
           "-o", str(exe)]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0, out.stdout + out.stderr
    rc = int(out.stdout.split()[1])
    import torch
    if not torch.cuda.is_available():
        assert rc != api.OK


def test_init_fails_cleanly_without_gpu():
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    with pytest.raises(api.PtbGpuError):
        api.Context(0)


class _NoCalls:
    """Stands in for the loaded library: any C call fails the test."""

    def __getattr__(self, name):
        raise AssertionError(f"{name} was called with arrays of the wrong length")


def _unbound_context():
    ctx = api.Context.__new__(api.Context)
    ctx._lib, ctx._h, ctx.device = _NoCalls(), None, 0
    return ctx


def test_wrong_array_lengths_are_rejected_before_the_c_call():
    import numpy as np
    ctx = _unbound_context()
    n, nat = 10, 4
    pk, short = np.zeros(n * (n + 1) // 2), np.zeros(n * (n + 1) // 2 - 1)
    aoat, xyz = np.repeat(np.arange(1, nat + 1), [3, 3, 2, 2]), np.zeros((nat, 3))
    calls = [
        lambda: ctx.filter_matrix_sym(short, n, 1e-5),
        lambda: ctx.check_density(n, pk, short),
        lambda: ctx.check_density(n, pk, pk, short),
        lambda: ctx.sm_stupid_simple(n, 8, short, pk, nat, xyz, aoat, 2, 2),
        lambda: ctx.sm_stupid_simple(n, 8, pk, pk, nat, xyz[:3], aoat, 2, 2),
        lambda: ctx.sm_stupid_simple(n, 8, pk, pk, nat, xyz, aoat[:-1], 2, 2),
        lambda: ctx.sm_plan(n, pk, short, nat, xyz, aoat, 2, 2),
        lambda: ctx.kmeans_partition(n, pk, pk, nat, xyz, aoat[1:]),
        lambda: ctx.purification(api.PurificationSettings(), n, pk, short),
        lambda: ctx.tc_purify(n, 8, short, pk),
        lambda: ctx.tc_purify(n + 1, 8, pk, pk),
        lambda: ctx.tc_purify_batch([(n, 8, pk, pk), (n, 8, pk, short)]),
        lambda: ctx.tc_purify_grouped([(n, 8, short, pk)]),
        lambda: ctx.eig_density_batch([(n, 8, pk, pk), (n, 8, short, pk)]),
        lambda: ctx.eig_density_batch([(n, 8, pk, pk), (n, 7, pk, pk)]),
        lambda: ctx.solve2(1, n, 8, 0, pk, short),
        lambda: ctx.mlpop14(n, short),
        lambda: ctx.mlpop2(nat, n, short, np.eye(n), np.eye(n), aoat, aoat),
        lambda: ctx.mlpop2(nat, n, pk, np.eye(n - 1), np.eye(n), aoat, aoat),
        lambda: ctx.mlpop2(nat, n, pk, np.eye(n), np.eye(n), aoat, aoat[:-2]),
        lambda: ctx.xc_damping(nat, n, aoat, np.zeros(10), np.zeros(nat), np.zeros(n), np.zeros(n), short, pk),
        lambda: ctx.xc_damping(nat, n, aoat, np.zeros(9), np.zeros(nat), np.zeros(n), np.zeros(n), pk, pk),
        lambda: ctx.xc_damping_device(nat, n, aoat, np.zeros(10), np.zeros(nat + 1), np.zeros(n), np.zeros(n), 0, 0),
    ]
    for k, call in enumerate(calls):
        with pytest.raises(api.PtbGpuError) as ei:
            call()
        assert ei.value.code == api.EINVAL, k


def test_output_arrays_are_checked_before_the_c_call():
    """A caller-provided P (e.g. in pinned memory) must be contiguous float64
    of npacked(ndim) elements."""
    import numpy as np
    ctx = _unbound_context()
    n, nat = 10, 4
    npk = n * (n + 1) // 2
    pk = np.zeros(npk)
    aoat, xyz = np.repeat(np.arange(1, nat + 1), [3, 3, 2, 2]), np.zeros((nat, 3))
    bad = [np.zeros(npk - 1), np.zeros(npk, dtype=np.float32), np.zeros(2 * npk)[::2]]
    for out in bad:
        with pytest.raises(ValueError):
            ctx.sm_stupid_simple(n, 8, pk, pk, nat, xyz, aoat, 2, 2, out=out)
        with pytest.raises(ValueError):
            ctx.tc_purify(n, 8, pk, pk, out=out)


FORTRAN_MODULE = HEADER.parent / "ptbgpu_c.f90"
FORTRAN_SHIMS = HEADER.parent / "ptbgpu_shims.f90"


def _fortran_fields(name):
    """Field list of a bind(C) derived type in the Fortran module include/ptbgpu_c.f90."""
    src = FORTRAN_MODULE.read_text()
    m = re.search(r"type, bind\(C\) :: " + name + r"\b[^\n]*\n(.*?)end type", src, re.S)
    assert m, name
    out = []
    for line in m.group(1).splitlines():
        mm = re.match(r"\s*(real\(c_double\)|integer\(c_int64_t\))\s*::\s*(.*)", line.split("!")[0])
        if mm:
            kind = "double" if mm.group(1).startswith("real") else "int64_t"
            out += [(kind, v.split("=")[0].strip()) for v in mm.group(2).split(",")]
    return out


@pytest.mark.parametrize("name", ["ptbgpu_opts", "ptbgpu_stats", "ptbgpu_pur_settings"])
def test_fortran_binding_types_match_header(name):
    """The bind(C) types of include/ptbgpu_c.f90 have the header's fields in the
    header's order and kinds (a mismatch would shift every later field of the
    struct the library writes)."""
    text = HEADER.read_text()
    m = re.search(r"typedef struct \{([^{}]*)\}\s*" + name + ";", text)
    body = re.sub(r"/\*.*?\*/", "", m.group(1), flags=re.S)
    c_fields = re.findall(r"\b(int64_t|double)\s+(\w+)\s*;", body)
    assert _fortran_fields(name) == c_fields


def test_fortran_interfaces_bind_declared_exports():
    """Every bind(C, name=...) interface of the Fortran module names a function the
    header declares and the library exports, with as many dummy arguments as the
    C prototype has parameters; every function the shims call is bound."""
    src = FORTRAN_MODULE.read_text()
    header = HEADER.read_text()
    lib = api.load_library()
    binds = re.findall(r"function\s+(ptbgpu_\w+)\s*\(([^)]*)\)[^\n]*?(?:&\s*\n\s*)?[^\n]*?bind\(C, name=\"(\w+)\"\)",
                       src, re.S)
    assert len(binds) >= 6
    for fname, dummies, cname in binds:
        assert fname == cname
        assert hasattr(lib, cname), cname
        proto = re.search(r"\b" + cname + r"\s*\(([^)]*)\)\s*;", header)
        assert proto, cname
        n_c = len([a for a in proto.group(1).split(",") if a.strip() and a.strip() != "void"])
        n_f = len([a for a in dummies.replace("&", " ").split(",") if a.strip()])
        assert n_f == n_c, (cname, n_f, n_c)
    bound = {c for _, _, c in binds}
    called = set(re.findall(r"\b(ptbgpu_[a-z0-9_]+)\s*\(", FORTRAN_SHIMS.read_text()))
    called -= {"ptbgpu_pur_settings"}   # the derived type's structure constructor
    assert called and called <= bound, called - bound
