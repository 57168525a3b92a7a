"""The C ABI library (no GPU needed): it loads, exports every entry point the
headers in include/ declare, and rejects bad arguments with a status code
instead of aborting."""
import ctypes
import os
import re

import pytest

from a5_streamer_b200 import _lib, build

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared():
    names = []
    for h in ("a5g.h", "a5t.h", "a5g3.h", "a5a.h"):
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^\s*(?:const\s+)?\w+\s*\*?\s*(a5(?:[gtsa]|g3)_\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_library_builds_and_loads():
    build.build()
    assert _lib.lib().a5g_version() == 1


def test_every_declared_symbol_is_exported():
    names = declared()
    assert len(names) > 40
    L = _lib.lib()
    missing = [n for n in names if not hasattr(L, n)]
    assert not missing, missing
    # the Python binding covers the whole ABI
    assert set(names) <= set(_lib.SIGNATURES), set(names) - set(_lib.SIGNATURES)


def test_invalid_parameters_are_rejected_without_a_device():
    p = _lib.Params()
    p.box_size = 16  # only 8 is built
    p.lvls_max = 7
    p.dr_base = 1.0
    h = ctypes.c_void_p()
    code = _lib.lib().a5g_create(ctypes.byref(p), ctypes.byref(h))
    assert code == _lib.A5G_EINVAL
    assert b"box_size" in _lib.lib().a5g_last_error()
    p.box_size = 8
    p.epsilon_diel = 0.0  # a permittivity must be positive
    assert _lib.lib().a5g_create(ctypes.byref(p), ctypes.byref(h)) == _lib.A5G_EINVAL
    # null arguments
    assert _lib.lib().a5g_step(None, 1e-12) == _lib.A5G_EINVAL
    assert _lib.lib().a5g_step_batch(None, 0, None) == _lib.A5G_EINVAL


def test_adjoint_rejects_bad_arguments_without_a_device():
    L = _lib.lib()
    ap = _lib.AdjParams(200, 20, 4e-3, 1.0)
    h = ctypes.c_void_p()
    dts = (ctypes.c_double * 200)(*([1e-12] * 200))
    assert L.a5a_create(None, ctypes.byref(ap), dts, ctypes.byref(h)) == _lib.A5G_EINVAL
    assert L.a5a_forward(None, None) == _lib.A5G_EINVAL
    assert L.a5a_gradient(None, None, None, None) == _lib.A5G_EINVAL
    assert L.a5a_destroy(None) == _lib.A5G_OK
    sizes = (ctypes.c_longlong * 4)()
    one = (ctypes.c_int * 16)()
    geo = (ctypes.c_double * 4)()
    cnt = (ctypes.c_int * 3)()
    ids = (ctypes.c_int * 1)()
    # a segment outside 0..8
    assert L.a5a_debug_tape(0, 1, 1, one, geo, cnt, ids, 1, 8, 9, sizes,
                            None, None, None, None, None, None) == _lib.A5G_EINVAL
    assert b"segment" in L.a5g_last_error()


def _fortran_params_layout():
    """Field offsets and size of the Fortran a5g_params_t documented in
    INTEGRATION.md, by the C layout rules a bind(C) type follows (c_int: 4
    bytes, c_double: 8 bytes, each aligned to its size; arrays contiguous)."""
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    body = re.search(r"type, bind\(C\) :: a5g_params_t\n(.*?)\n\s*end type a5g_params_t", text, re.S)
    assert body, "a5g_params_t not found in INTEGRATION.md"
    sizes = {"integer(c_int)": 4, "real(c_double)": 8}
    fields, off, align = [], 0, 1
    for line in body.group(1).splitlines():
        kind, decl = [x.strip() for x in line.split("::")]
        size = sizes[kind]
        for item in re.findall(r"(\w+)(\([^)]*\))?", decl):
            name, dims = item
            n = 1
            for d in re.findall(r"\d+", dims):
                n *= int(d)
            off = (off + size - 1) // size * size
            fields.append((name, off))
            off += n * size
            align = max(align, size)
    return fields, (off + align - 1) // align * align


def test_params_layout_documented_python_and_c_agree():
    """The Fortran binding in INTEGRATION.md, the ctypes mirror and the C
    struct the library was compiled with have the same fields at the same
    offsets and the same size: a caller following any of them passes the
    object a5g_create reads."""
    fields, size = _fortran_params_layout()
    names = [f for f, _ in _lib.Params._fields_]
    assert [f for f, _ in fields] == names
    for name, off in fields:
        assert getattr(_lib.Params, name).offset == off, name
    assert ctypes.sizeof(_lib.Params) == size
    out = (ctypes.c_int * 64)()
    n = _lib.lib().a5g_debug_params_layout(out, 64)
    assert n == 1 + len(names)
    assert out[0] == size
    assert list(out[1:n]) == [off for _, off in fields]


def test_error_raises_with_status_name():
    with pytest.raises(_lib.A5GError) as e:
        _lib.call("a5g_step", None, 1e-12)
    assert "A5G_EINVAL" in str(e.value)


def test_new_entry_points_reject_bad_arguments_without_a_device():
    L = _lib.lib()
    E = _lib.A5G_EINVAL
    # precision of a missing context, or an unknown precision
    assert L.a5g_set_precision(None, 1, None) == E
    assert L.a5g_get_precision(None, None, None) == E
    # device-driven batch: null or empty member lists, null batch handles
    out = ctypes.c_void_p()
    assert L.a5g_batch_create(None, 1, ctypes.byref(out)) == E
    assert L.a5g_batch_create(None, 0, ctypes.byref(out)) == E
    assert L.a5g_batch_begin(None, None, None) == E
    assert L.a5g_batch_block(None, 2, 1, None, None, None, None) == E
    assert L.a5g_batch_launch(None, 2, 1) == E
    assert L.a5g_batch_finish(None, None, None, None, None) == E
    assert L.a5g_batch_destroy(None) == _lib.A5G_OK
    # batched driver: no members, bad group count
    assert L.a5s_batch_run(None, 0, None, 1, 1, 1, 1, None, None, None, None) == E
    arr = (ctypes.c_void_p * 1)(None)
    te = (ctypes.c_double * 1)(1e-9)
    assert L.a5s_batch_run(arr, 1, te, 1, 1, 0, 1, None, None, None, None) == E
    assert L.a5s_batch_run(arr, 1, te, 1, 1, 1, 1, None, None, None, None) == E  # null member
    # the allocation-free batch: null member list
    assert L.a5g_step_batch_static(None, 1, None) == E
    # checkpoint / resume: null run or buffer
    n = ctypes.c_size_t(0)
    assert L.a5s_checkpoint_size(None, ctypes.byref(n)) == E
    assert L.a5s_checkpoint_save(None, None, 0, None) == E
    assert L.a5s_checkpoint_load(None, b"A5CK", 4) == E
