"""Argument checks of the C ABI that happen on the host before any device work, so
they run without a GPU: each invalid call returns RQ_E_INVALID (-1) with the
reference's message, as the reference raises ValueError / std::invalid_argument."""
import ctypes as C

import numpy as np

import rans_uq_b200._native as N


def err(L):
    return L.rq_last_error().decode()


def test_statistics_entry_points_reject_what_the_reference_rejects(rq):
    L = rq.lib()
    w = np.array([0.5, 0.6])
    u = np.array([0.1])
    idx = np.zeros(1, dtype=np.int64)
    ip = idx.ctypes.data_as(C.POINTER(C.c_int64))
    assert L.rq_resample_indices(N.dptr(w), 2, N.dptr(u), 1, ip) == -1
    assert "sum to 1" in err(L)
    w = np.array([1.5, -0.5])
    assert L.rq_resample_indices(N.dptr(w), 2, N.dptr(u), 1, ip) == -1
    assert "non-negative" in err(L)
    w = np.array([0.5, 0.5])
    u = np.array([1.0])  # uniforms lie in [0, 1)
    assert L.rq_resample_indices(N.dptr(w), 2, N.dptr(u), 1, ip) == -1
    q = C.c_double()
    s = np.array([1.0, -2.0])
    assert L.rq_conformal_quantile(N.dptr(s), 2, C.c_double(0.1), C.byref(q)) == -1
    assert "nonnegative" in err(L)
    s = np.array([1.0, 2.0])
    for alpha in (0.0, 1.0, float("nan")):
        assert L.rq_conformal_quantile(N.dptr(s), 2, C.c_double(alpha), C.byref(q)) == -1
        assert "alpha" in err(L)
    s = np.array([1.0, np.inf])
    assert L.rq_conformal_quantile(N.dptr(s), 2, C.c_double(0.1), C.byref(q)) == -1
    assert "finite" in err(L)
    x = np.array([[1.0, np.nan]])
    m, v = np.zeros(2), np.zeros(2)
    assert L.rq_predictive_moments(N.dptr(x), 1, 2, N.dptr(m), N.dptr(v)) == -1
    assert L.rq_predictive_moments(N.dptr(x), 0, 2, N.dptr(m), N.dptr(v)) == -1
    ll = np.array([-1.0])
    assert L.rq_posterior_weights_parts(N.dptr(ll), None, 0, N.dptr(m), N.dptr(m),
                                        N.dptr(m)) == -1


def test_warm_cache_and_model_entry_points_check_arguments(rq):
    L = rq.lib()
    out = C.c_void_p()
    assert L.rq_warm_cache_create(None, 50, C.c_double(0.5), 1 << 26, C.byref(out)) == -1
    assert "null" in err(L)
    row = N.RowOut()
    theta = np.array([0.31, 0.09])
    assert L.rq_evaluate_cached(None, N.dptr(theta), C.byref(row), None, None, None, None,
                                None, None) == -1
    size = C.c_int32()
    assert L.rq_warm_cache_info(None, C.byref(size), None, None) == -1
    assert L.rq_warm_cache_clear(None) == -1
    assert L.rq_warm_cache_set_byte_budget(None, 0) == -1
    assert L.rq_warm_cache_destroy(None) == 0  # deleting nothing is allowed, as delete is
    assert L.rq_mesh_save_binary(None, b"x") == -1


def test_version_is_reported(rq):
    assert rq.lib().rq_version() > 0


def test_missing_library_fails_loudly(tmp_path):
    """Without the built CUDA library every call raises: there is no CPU path."""
    import subprocess
    import sys
    from pathlib import Path

    root = Path(__file__).resolve().parents[1]
    code = (
        "import sys; sys.path.insert(0, %r)\n"
        "import rans_uq_b200._native as N\n"
        "from pathlib import Path\n"
        "N.LIB_PATH = Path(%r)\n"
        "import rans_uq_b200 as rq\n"
        "try:\n"
        "    rq.Mesh.make_periodic_channel_2d(3, 8, 1.0, 1.0, 180.0, 1.0).cell_geometry()\n"
        "except ImportError as e:\n"
        "    print('raised', e)\n"
    ) % (str(root), str(tmp_path / "absent.so"))
    out = subprocess.run([sys.executable, "-c", code], capture_output=True, text=True,
                         timeout=120)
    assert "raised" in out.stdout and "no CPU fallback" in out.stdout, out.stdout + out.stderr
