"""Host-side argument checks of the serving, progressive-estimation and cache
snapshot entry points.  Each check fails with N2W_EINVAL and a message before
any CUDA call, so these run without a GPU."""
import ctypes as C

import numpy as np


def _status(lib, name, *args):
    st = getattr(lib, name)(*args)
    return st, lib.n2w_last_error().decode()


def test_server_option_defaults(n2w):
    from n2w._lib import ServerOptions, call

    o = ServerOptions()
    call("n2w_server_options_default", C.byref(o))
    assert (o.pool_bytes, o.max_inflight, o.tick_walks, o.max_steps) == (0, 256, 1 << 21, 256)
    assert abs(o.pool_fraction - 0.25) < 1e-7 and abs(o.epsilon - 1e-3) < 1e-9
    assert (o.block_size, o.regen_threshold, o.chunk, o.tick_walks_max) == (256, 8, 1, 1 << 23)


def test_server_create_rejects_bad_options(n2w):
    from n2w._lib import Problem, ServerOptions, call, lib

    bvhs = (C.c_void_p * 1)(None)
    probs = (Problem * 1)(n2w.problem_charges_seeded())
    out = C.c_void_p()
    for field, value, needle in (("chunk", 65, "chunk"), ("max_inflight", 0, "max_inflight"),
                                 ("tick_walks", 16, "tick_walks"), ("block_size", 48, "block_size"),
                                 ("epsilon", 0.0, "walk options"), ("tick_walks_max", -1, "tick_walks_max")):
        o = ServerOptions()
        call("n2w_server_options_default", C.byref(o))
        setattr(o, field, value)
        st, msg = _status(lib, "n2w_server_create", bvhs, 1, probs, 1, C.byref(o), C.byref(out))
        assert st == 1 and needle in msg, (field, st, msg)
        assert not out.value
    st, msg = _status(lib, "n2w_server_create", None, 1, probs, 1, None, C.byref(out))
    assert st == 1 and "bad arguments" in msg


def test_server_calls_reject_null_server(n2w):
    from n2w._lib import Request, ServerNc, lib

    nc = ServerNc()
    st, msg = _status(lib, "n2w_server_set_nc", None, 0, 0, C.byref(nc))
    assert st == 1 and "null" in msg
    r = Request()
    rid = C.c_int64()
    pts = np.zeros(3, np.float32)
    st, msg = _status(lib, "n2w_server_submit", None, C.byref(r), pts.ctypes.data_as(C.c_void_p), C.byref(rid))
    assert st == 1 and "null" in msg


def test_progressive_and_snapshot_copy_reject_null_arguments(n2w):
    from n2w._lib import NcProgressiveOptions, PointStats, lib

    o = NcProgressiveOptions()
    o.blocks = 2
    empty = PointStats()
    st, msg = _status(lib, "n2w_nc_progressive", None, None, None, None, None, 0, C.byref(o), empty, empty, None,
                      None, None)
    assert st == 1 and "null argument" in msg
    st, msg = _status(lib, "n2w_cache_copy_params", None, None, None)
    assert st == 1 and "null argument" in msg
