"""C-ABI checks that need no GPU: the library loads, exports every symbol the
header declares, and rejects bad arguments before touching the device."""
import ctypes as C

import pytest

from ginkgo_b200 import _lib


def test_library_exports_every_declared_symbol():
    lib = _lib.lib()
    declared = _lib.declared_symbols()
    assert len(declared) >= 20
    missing = [n for n in declared if not hasattr(lib, n)]
    assert not missing, missing
    assert lib.b2s_version() == 1


def test_load_balance_tile_count():
    lib = _lib.lib()
    # 34 words per 256-entry chunk (at least one chunk) + 4, minus one
    assert lib.b2s_csr_load_balance_num_tiles(0, 0) == 37
    assert lib.b2s_csr_load_balance_num_tiles(2048, 0) == 37
    assert lib.b2s_csr_load_balance_num_tiles(10, 257) == 34 * 2 + 3
    assert lib.b2s_csr_load_balance_num_tiles(2097152, 14581760) == \
        34 * ((14581760 + 255) // 256) + 3
    assert lib.b2s_csr_load_balance_num_tiles(-1, 0) == -1


def _spmv(**kw):
    args = dict(strategy=0, n=4, m=4, rp=None, ci=None, v=None, mrn=1,
                tiles=None, nt=0, b=None, ldb=1, c=None, ldc=1, k=1,
                alpha=None, beta=None)
    args.update(kw)
    return _lib.lib().b2s_csr_spmv_f64(*args.values(), None)


def test_spmv_rejects_bad_arguments_without_device_work():
    lib = _lib.lib()
    fake = C.c_void_p(16)  # never dereferenced: validation fails first
    assert _spmv(strategy=7, rp=fake, b=fake, c=fake) == -1
    assert b"strategy" in lib.b2s_last_error()
    assert _spmv(alpha=fake, rp=fake, b=fake, c=fake) == -1
    assert b"alpha and beta" in lib.b2s_last_error()
    assert _spmv(k=3, ldb=2, ldc=3, rp=fake, b=fake, c=fake) == -1
    assert _spmv(strategy=1, rp=fake, b=fake, c=fake) == -1
    assert b"partition" in lib.b2s_last_error()
    # a partition size that b2s_csr_load_balance_num_tiles cannot return
    assert _spmv(strategy=1, rp=fake, b=fake, c=fake, tiles=fake, nt=40) == -1
    assert b"partition" in lib.b2s_last_error()
    # empty work is a no-op that needs no device
    assert _spmv(n=0) == 0
    assert _spmv(k=0) == 0


def test_workspace_queries():
    lib = _lib.lib()
    assert lib.b2s_sellp_slice_sets_workspace_bytes(100, 0) == -1
    assert lib.b2s_sellp_slice_sets_workspace_bytes(100, 32) >= 16
    assert lib.b2s_csr_transpose_workspace_bytes(10, 10, 30, 8) >= 30 * 12


def test_ell_rejects_short_stride():
    lib = _lib.lib()
    fake = C.c_void_p(16)
    rc = lib.b2s_ell_spmv_f64(10, 10, 3, 5, fake, fake, fake, 1, fake, 1, 1,
                              None, None, None)
    assert rc == -1 and b"stride" in lib.b2s_last_error()


def test_missing_library_fails_loudly(monkeypatch, tmp_path):
    monkeypatch.setattr(_lib, "_lib", None)
    monkeypatch.setattr(_lib, "LIB_PATH", str(tmp_path / "absent.so"))
    import ginkgo_b200.build as b
    monkeypatch.setattr(b, "build", lambda *a, **k: (_ for _ in ()).throw(
        RuntimeError("nvcc not available")))
    with pytest.raises(RuntimeError):
        _lib.lib()
