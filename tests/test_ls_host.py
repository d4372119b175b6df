"""CPU: the ls handle is host state -- memLS_LS_CREATE's defaults and
arguments, the precision switch and the log path are set and checked
without a GPU."""
import ctypes

import numpy as np

from crimsonflowsolver_b200 import _native as N


def test_ls_create_settings_without_gpu(tmp_path):
    L = N.lib()
    ls = ctypes.c_void_p()
    rin = np.array([1e-4, 1e-4])
    ain = np.array([1e-10, 1e-10])
    min_ = np.array([10, 500], dtype=np.int32)
    rc = L.crimson_memls_ls_create(ctypes.byref(ls), 3, 1 | 4 | 8 | 16 | 64, 1e-5, 0.0, 10, 50, N.dp(rin), N.dp(ain),
                                   N.ip(min_))
    assert rc == N.OK
    bad = ctypes.c_void_p()
    assert L.crimson_memls_ls_create(ctypes.byref(bad), 2, 0, 0.0, 0.0, 0, 0, None, None, None) == 2  # UNSUPPORTED
    try:
        assert L.crimson_memls_ls_set_precision(ls, 1, 8, 0.0) == N.OK
        assert L.crimson_memls_ls_set_precision(ls, 3, 8, 0.0) == 1          # unknown mode: CRIMSON_ERR_ARG
        assert L.crimson_memls_ls_set_log(ls, str(tmp_path / "memLS_NS.log").encode()) == N.OK
        assert L.crimson_memls_ls_set_log(ls, None) == N.OK
        assert L.crimson_memls_ls_set_log(None, None) == 1
        assert not (tmp_path / "memLS_NS.log").exists()                    # nothing written before a solve
    finally:
        L.crimson_memls_ls_free(ls)
