"""The C ABI loads on a machine without a GPU and exports every entry point
that include/gsw.h declares; calls without a device fail with a status code,
never a crash or a silent fallback."""
import ctypes
import os
import re

import pytest

import gswitch_b200 as gs

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    txt = open(os.path.join(ROOT, "include", "gsw.h")).read()
    txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
    return sorted(set(re.findall(r"\b(gsw_[a-z_0-9]+)\s*\(", txt)))


@pytest.fixture(scope="module")
def lib():
    from gswitch_b200 import build

    build.build()
    return ctypes.CDLL(gs.LIB_PATH)


def test_every_declared_symbol_is_exported(lib):
    syms = declared_symbols()
    assert len(syms) >= 20
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing
    assert set(syms) == set(gs.ABI_SYMBOLS)


def test_version_and_defaults(lib):
    L = gs.lib()
    assert L.gsw_version() == 1
    o = gs._Opts()
    L.gsw_run_opts_default(ctypes.byref(o))
    assert (o.direction, o.asfmt, o.lb, o.fusion) == (-1, -1, -1, -1)
    assert o.sorted_queue == 1 and abs(o.damping - 0.85) < 1e-7


def test_config_string_parsing():
    o = gs.RunOpts.from_config("Pull-Bitmap-STRICT-Standalone")
    assert (o.direction, o.asfmt, o.lb, o.fusion) == (gs.PULL, gs.BITMAP, 3, gs.STANDALONE)
    o = gs.RunOpts.from_config("x-Queue")
    assert (o.direction, o.asfmt, o.lb, o.fusion) == (None, gs.QUEUE, None, None)


def test_init_reports_status_without_device():
    import torch

    if torch.cuda.is_available():
        pytest.skip("a device is present")
    with pytest.raises(gs.GswError) as e:
        gs.Context(0)
    assert e.value.code in (3, 7)


def test_caller_driven_loop_rejects_null_handles(lib):
    """The level-loop entry points check their handles before touching a
    device: NULL context, graph or traversal is INVALID_ARG."""
    L = gs.lib()
    t = ctypes.c_void_p()
    assert L.gsw_traversal_begin(None, None, gs.APP_BFS, 0, None, ctypes.byref(t)) == 1
    st = gs.LevelStats()
    done = ctypes.c_int(0)
    assert L.gsw_level_begin(None, ctypes.byref(st), ctypes.byref(done)) == 1
    ch = gs.LevelChoice(gs.PUSH, gs.QUEUE, 0, 0)
    assert L.gsw_level_end(None, ctypes.byref(ch)) == 1
    assert L.gsw_traversal_end(None, None, None) == 1
    assert L.gsw_select(None, ctypes.byref(st), 0, ctypes.byref(ch)) == 1
