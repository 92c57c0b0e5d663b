"""Host-side logic that needs no GPU: generators, batch layout, factory
parameters, the conductivity assembly used by the differentiable solve."""
import numpy as np
import pytest
import torch

from ginkgo_b200 import stencils
from oracle import oracle as orc


def test_generator_sizes_match_the_workloads():
    assert len(stencils.poisson_2d_5pt(256)[1]) == 326656
    rp, ci, _ = stencils.poisson_3d_7pt(64)
    assert (len(rp) - 1, len(ci)) == (262144, 1810432)
    rp, ci, v = stencils.anisotropic_27pt(8)
    n = len(rp) - 1
    # symmetric, positive definite
    dense = np.zeros((n, n))
    dense[np.repeat(np.arange(n), np.diff(rp)), ci] = v
    assert np.allclose(dense, dense.T)
    assert np.linalg.eigvalsh(dense).min() > 0


def test_power_law_rows_sorted_and_unique():
    rp, ci, v = stencils.power_law(5000, seed=1, max_len=800)
    for r in range(0, 5000, 97):
        row = ci[rp[r]:rp[r + 1]]
        assert np.all(np.diff(row) > 0)
    assert rp[-1] == len(ci) == len(v)


def test_std_uniform_reproduces_mt19937():
    # first outputs of std::mt19937(5489) are 3499211612, 581869302
    w = np.frombuffer(np.random.RandomState(5489).bytes(8), "<u4")
    assert list(w) == [3499211612, 581869302]
    u = stencils.std_uniform(5489, 1, 0.0, 1.0)[0]
    assert u == (3499211612 + 581869302 * 2.0 ** 32) / 2.0 ** 64


def test_batch_ell_layout_matches_per_system_ell():
    from ginkgo_b200.batch import BatchEll

    class FakeExec:
        device = torch.device("cpu")

    systems = [stencils.convection_diffusion_2d(nx, ny, 1.0, 0.3, -0.2)
               for nx, ny in ((5, 4), (7, 3), (1, 9))]
    A = BatchEll.from_csr(FakeExec(), systems, width=5)
    ci = A.col_idxs.numpy()
    v = A.values.numpy()
    for s, (rp, c, val) in enumerate(systems):
        w, st, eci, ev = orc.csr_to_ell(rp, c, val, width=5)
        o = 5 * A.host_row_offsets[s]
        assert np.array_equal(ci[o:o + len(eci)], eci)
        assert np.array_equal(v[o:o + len(ev)], ev)
    back = A.to_csr_list()
    for (rp, c, val), (rp2, c2, v2) in zip(systems, back):
        assert np.array_equal(rp, rp2) and np.array_equal(c, c2)
        assert np.allclose(val, v2)


def test_conductivity_assembly_matches_generator():
    from ginkgo_b200.autograd import ConductivityOperator
    op = ConductivityOperator(5, device="cpu")
    th = torch.rand(op.num_edges, dtype=torch.float64) + 0.25
    rp, ci, v = stencils.conductivity_matrix(5, th.numpy())
    assert np.array_equal(op.row_ptrs.numpy(), rp)
    assert np.array_equal(op.col_idxs.numpy(), ci)
    assert np.allclose(op.values(th).numpy(), v)
    # gradient of sum(values) w.r.t. theta: interior edges 2 - 2 = 0, boundary 1
    th.requires_grad_(True)
    op.values(th).sum().backward()
    ei, ej = stencils.conductivity_edges(5)
    assert np.allclose(th.grad.numpy(), np.where(ej >= 0, 0.0, 1.0))


def test_solver_factory_parameters():
    from ginkgo_b200.solver import (Cg, Gmres, Iteration, Jacobi, ResidualNorm,
                                    _criteria)
    m, r, mode = _criteria((Iteration.build().with_max_iters(50),
                            ResidualNorm.build().with_reduction_factor(1e-8)))
    assert (m, r, mode) == (50, 1e-8, 0)
    with pytest.raises(ValueError):
        _criteria((ResidualNorm.build().with_reduction_factor(1e-8),))
    # baselines and the implicit norm map to the C ABI's residual modes
    from ginkgo_b200.solver import ImplicitResidualNorm
    it = Iteration.build().with_max_iters(5)
    for base, code in (("rhs_norm", 0), ("initial_resnorm", 1), ("absolute", 2)):
        assert _criteria((it, ResidualNorm.build().with_baseline(base)))[2] == code
        assert _criteria((it, ImplicitResidualNorm.build().with_baseline(base)))[2] == code | 4
    with pytest.raises(ValueError):
        ResidualNorm.build().with_baseline("relative").on(None)
    with pytest.raises(NotImplementedError):
        _criteria((it, ResidualNorm.build(), ImplicitResidualNorm.build()))
    assert Jacobi.build().with_max_block_size(4).on(None).max_block_size == 4
    # the reference's GMRES defaults: krylov_dim 100, modified Gram-Schmidt
    f = Gmres.build().with_criteria(it).on(None)
    assert f.krylov_dim == 100 and f.ortho_method == "mgs"
    f = Gmres.build().with_krylov_dim(300).with_criteria(it).on(None)
    assert f.krylov_dim == 300  # not changed here; the device rejects it
    with pytest.raises(ValueError):
        Gmres.build().with_ortho_method("householder").with_criteria(it).on(None)
    f = Cg.build().with_criteria(Iteration.build().with_max_iters(3)).on(None)
    assert f.kind == "cg" and f.max_iters == 3 and f.reduction == 0.0


def test_gmres_workspace_query_rejects_unsupported_krylov_dims():
    from ginkgo_b200._lib import lib
    q = lib().b2s_gmres_workspace_bytes
    assert q(1000, 5000, 7, 1, 128, 0) > 0
    assert q(1000, 5000, 7, 4, 100, 3) > 0
    assert q(1000, 5000, 7, 1, 129, 0) == -1
    assert q(1000, 5000, 7, 1, 0, 0) == -1
    assert q(1000, 5000, 7, 1, 30, 9) == -1


def test_block_detection_matches_the_oracle():
    import json
    import os

    from ginkgo_b200.solver import find_blocks
    from oracle import jacobi as J
    here = os.path.dirname(os.path.abspath(__file__))
    with open(os.path.join(here, "golden", "jacobi_cases.json")) as f:
        cases = json.load(f)["blocks"]
    for c in cases:
        if "block_ptrs" in c:
            continue
        m = c["matrix"]
        got = find_blocks(m["row_ptrs"], m["col_idxs"], c["max_block_size"])
        assert got.tolist() == c["expected"], c["name"]
    rng = np.random.default_rng(0)
    for _ in range(30):
        # runs of rows sharing a pattern, of random lengths
        n, rows = 0, []
        while n < 300:
            run = int(rng.integers(1, 12))
            cols = np.sort(rng.choice(400, size=int(rng.integers(1, 6)), replace=False))
            rows += [cols] * run
            n += run
        rp = np.concatenate([[0], np.cumsum([len(r) for r in rows])])
        ci = np.concatenate(rows)
        for mbs in (1, 3, 8, 32):
            assert find_blocks(rp, ci, mbs).tolist() == J.find_blocks(rp, ci, mbs)


def test_hybrid_config_matches_the_oracle():
    from ginkgo_b200.matrix import hybrid_config
    from oracle import spgemm as S
    # the reference's own cases (core/test/matrix/hybrid.cpp:170-244)
    assert hybrid_config([3, 1], "automatic") == (0, 4)
    assert hybrid_config([3, 2], "column_limit", num_columns=2) == (2, 1)
    assert hybrid_config([3, 1], "imbalance_limit", percent=0.4) == (1, 2)
    assert hybrid_config([], "automatic") == (0, 0)
    rng = np.random.default_rng(2)
    cases = [("automatic", {}), ("imbalance_limit", {"percent": 0.3}),
             ("imbalance_limit", {"percent": 1.0}), ("imbalance_limit", {"percent": 1.7}),
             ("imbalance_bounded_limit", {"percent": 0.9, "ratio": 0.02}),
             ("minimal_storage_limit", {}), ("column_limit", {"num_columns": 5})]
    for _ in range(25):
        lens = rng.integers(0, 40, size=int(rng.integers(1, 3000)))
        for strat, kw in cases:
            w = S.hybrid_width(lens, strat, **kw)
            assert hybrid_config(lens, strat, **kw) == (w, int(np.maximum(lens - w, 0).sum()))
    with pytest.raises(ValueError):
        hybrid_config([1, 2], "column_limit")


def test_hybrid_config_rejects_bad_parameters():
    from ginkgo_b200.matrix import hybrid_config
    nan, inf = float("nan"), float("inf")
    bad = [("imbalance_bounded_limit", {"percent": 0.8, "ratio": -0.5}),
           ("imbalance_bounded_limit", {"percent": 0.8, "ratio": nan}),
           ("imbalance_bounded_limit", {"percent": 0.8, "ratio": inf}),
           ("imbalance_bounded_limit", {"percent": nan, "ratio": 0.1}),
           ("imbalance_limit", {"percent": nan}),
           ("column_limit", {"num_columns": nan}),
           ("column_limit", {"num_columns": inf}),
           ("column_limit", {"num_columns": -1}),
           ("column_limit", {"num_columns": 1e30})]
    for strat, kw in bad:
        with pytest.raises(RuntimeError):
            hybrid_config([3, 1, 4], strat, **kw)


def test_slice_sets_reject_null_pointers_before_device_work():
    import ctypes as C
    from ginkgo_b200 import _lib
    lib = _lib.lib()
    fake = C.c_void_p(256)  # never dereferenced: validation fails first
    # workspace form: null row_ptrs, then null slice_lengths
    assert lib.b2s_sellp_compute_slice_sets(64, None, 32, 1, fake, fake, fake,
                                            1 << 20, None) == -1
    assert lib.b2s_sellp_compute_slice_sets(64, fake, 32, 1, fake, None, fake,
                                            1 << 20, None) == -1
    assert b"null" in lib.b2s_last_error()
    # allocation-free form
    assert lib.b2s_sellp_compute_slice_sets_noalloc(64, None, 32, 1, fake, fake,
                                                    None) == -1
    assert lib.b2s_sellp_compute_slice_sets_noalloc(64, fake, 32, 1, fake, None,
                                                    None) == -1
    assert b"null" in lib.b2s_last_error()


def test_uniform_batch_ell_layout():
    from ginkgo_b200.batch import BatchEll

    class FakeExec:
        device = torch.device("cpu")

    rp, ci, v = stencils.convection_diffusion_2d(4, 3, 1.0, 0.2, -0.1)
    n = len(rp) - 1
    w, st, eci, ev = orc.csr_to_ell(rp, ci, v, width=5)
    vals = np.concatenate([ev, 2 * ev, 3 * ev])
    U = BatchEll.uniform(FakeExec(), 3, n, 5, torch.from_numpy(eci),
                         torch.from_numpy(vals))
    assert U.uniform_rows == n and U.total_rows == 3 * n
    back = U.to_csr_list()
    for s, (rp2, c2, v2) in enumerate(back):
        assert np.array_equal(rp2, rp) and np.array_equal(c2, ci)
        assert np.allclose(v2, (s + 1) * v)
    with pytest.raises(ValueError):
        BatchEll.uniform(FakeExec(), 3, n, 5, torch.from_numpy(eci[:-1]),
                         torch.from_numpy(vals))


def test_adaptive_jacobi_entries_reject_bad_arguments_before_device_work():
    import ctypes as C
    from ginkgo_b200 import _lib
    lib = _lib.lib()
    fake = C.c_void_p(256)  # never dereferenced: validation fails first
    nbytes = C.c_int64(0)
    assert lib.b2s_jacobi_adaptive_workspace_bytes(1000, C.byref(nbytes)) == 0
    assert nbytes.value == 4000  # one descriptor word per block
    assert lib.b2s_jacobi_adaptive_workspace_bytes(-1, C.byref(nbytes)) == -1
    # generation: conditioning, precisions, blocks and workspace are required
    args = [10, fake, fake, fake, 5, fake, 2, 0.1]
    assert lib.b2s_jacobi_block_generate_adaptive_f64(*args, None, fake, fake, 0, fake,
                                                      None) == -1
    assert lib.b2s_jacobi_block_generate_adaptive_f64(*args, fake, fake, fake, 0, None,
                                                      None) == -1
    assert lib.b2s_jacobi_block_generate_adaptive_f32(10, fake, fake, fake, 5, fake, 33, 0.1,
                                                      fake, fake, fake, 0, fake, None) == -1
    # apply without precisions, expand / reduce with a bad block size
    assert lib.b2s_jacobi_block_apply_adaptive_f64(10, 5, fake, 2, None, fake, fake, 1, fake,
                                                   1, 1, None, None, None) == -1
    assert lib.b2s_jacobi_block_expand_f64(5, 0, fake, fake, fake, None) == -1
    assert lib.b2s_jacobi_block_reduce_f32(5, 33, fake, fake, fake, None) == -1
    assert lib.b2s_jacobi_block_expand_f32(5, 4, None, fake, fake, None) == -1
