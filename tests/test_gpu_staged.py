"""Staged entry points (the reference's per-stage kernels and their tests:
tests/test_chol_n54.cpp, test_reduce_n54.cpp, test_reduce_eig_n54.cpp,
test_full_n54.cpp, and the finish kernel), the runtime-n solver's schedule
selection / autotune cache (test_autotune_n54.cpp, test_cache_n54.cpp,
test_cache_invalidation.cpp), and CUDA-graph capture."""
from __future__ import annotations

import os

import numpy as np
import pytest
import torch

import sbg
from oracle import metrics as Mx

pytestmark = pytest.mark.gpu

N = 54


@pytest.fixture(scope="module")
def pairs(oracle_mod):
    return oracle_mod.gen_fixture_pairs(N, 8, 42, "random")


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a)).cuda()


def test_chol_stage(pairs, oracle_mod):
    H, S = pairs
    Lr, _ = oracle_mod.potrf(S, N)
    for b in range(8):
        L = torch.empty((1, N * N), dtype=torch.complex128, device="cuda")
        info = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        sbg.chol_n54(dev(S[b:b + 1]), L, info)
        torch.cuda.synchronize()
        assert info.item() == 0
        L = L.cpu().numpy()
        # test_chol_n54.cpp:36: max-abs-diff / ||L||_F < 1e-12
        assert np.abs(L - Lr[b:b + 1]).max() / np.linalg.norm(Lr[b]) < 1e-12


def test_reduce_stage(pairs, oracle_mod):
    H, S = pairs
    Mr, _, _ = oracle_mod.reduce(H, S, N)
    for b in range(8):
        M = torch.empty((1, N * N), dtype=torch.complex128, device="cuda")
        info = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        sbg.reduce_n54(dev(H[b:b + 1]), dev(S[b:b + 1]), M, info)
        torch.cuda.synchronize()
        assert info.item() == 0
        # test_reduce_n54.cpp:39, 134-163: lower triangle, strict upper zeroed, < 1e-11
        assert np.abs(M.cpu().numpy() - Mr[b:b + 1]).max() < 1e-11 * max(1.0, np.abs(Mr[b]).max())


def test_reduce_eig_stage(pairs, oracle_mod):
    H, S = pairs
    Wr, Vr, _ = oracle_mod.reduce_eig(H, S, N)
    for b in range(8):
        W = torch.empty((1, N), dtype=torch.float64, device="cuda")
        V = torch.empty((1, N * N), dtype=torch.complex128, device="cuda")
        info = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        sbg.reduce_eig_n54(dev(H[b:b + 1]), dev(S[b:b + 1]), W, V, info)
        torch.cuda.synchronize()
        assert info.item() == 0
        W = W.cpu().numpy(); V = V.cpu().numpy()
        # test_reduce_eig_n54.cpp:14: eig 1e-10, 1 - |v_g^H v_r| < 1e-10 (Euclidean, V unitary)
        assert Mx.eig_rel_ref(W, Wr[b:b + 1]).max() < 1e-10
        I = np.eye(N).reshape(1, -1).astype(np.complex128)
        I = Mx.from_mats(np.eye(N)[None].astype(np.complex128))
        assert Mx.phase_err(I, V, Vr[b:b + 1], Wr[b:b + 1], N).max() < 1e-10


def test_full_single_stage(pairs, oracle_mod, golden_W):
    H, S = pairs
    for b in range(8):
        W = torch.empty((1, N), dtype=torch.float64, device="cuda")
        U = torch.empty((1, N * N), dtype=torch.complex128, device="cuda")
        info = torch.full((1,), -1, dtype=torch.int32, device="cuda")
        sbg.full_n54(dev(H[b:b + 1]), dev(S[b:b + 1]), W, U, info)
        torch.cuda.synchronize()
        assert info.item() == 0
        assert Mx.eig_rel_ref(W.cpu().numpy(), golden_W["n54_b8_s42_random"][b:b + 1]).max() < 1e-10


def test_finish_stage(pairs, oracle_mod):
    H, S = pairs
    M, L, _ = oracle_mod.reduce(H, S, N)
    Wr, Ur, _ = oracle_mod.finish(L, M, N)
    W = torch.empty((8, N), dtype=torch.float64, device="cuda")
    U = torch.empty((8, N * N), dtype=torch.complex128, device="cuda")
    info = torch.full((8,), -1, dtype=torch.int32, device="cuda")
    sbg.finish_n54(dev(L), dev(M), W, U, info, 8)
    torch.cuda.synchronize()
    assert (info.cpu().numpy() == 0).all()
    W = W.cpu().numpy(); U = U.cpu().numpy()
    assert Mx.eig_rel(W, Wr).max() < 1e-12
    assert Mx.phase_err(S, U, Ur, Wr, N).max() < 1e-10


def test_introspection_values():
    d = sbg.fixed_n54_introspection()
    assert d["geneig_full_n54_batched_block_dim_x"] in (128, 256)
    assert 0 < d["geneig_full_n54_batched_shared_mem_bytes"] <= 232448
    assert d["chol_n54_shared_mem_bytes"] > 0
    assert sbg.max_n("fp64") == 256 and 192 <= sbg.max_n("mixed") < 256


def test_solver_options_and_getters():
    s = sbg.Solver(32, batches_per_block=2, block_dim=128)
    assert s.batches_per_block == 2 and s.block_dim_x == 128
    assert s.cache_layer_used == "builtin" and not s.was_autotuned
    with pytest.raises(sbg.SolverError):
        sbg.Solver(32, block_dim=96)
    with pytest.raises(sbg.SolverError):
        sbg.Solver(sbg.max_n("fp64") + 1)
    with pytest.raises(sbg.SolverError):
        sbg.Solver(0)


def test_autotune_layers_and_corrupt_table(tmp_path, monkeypatch, oracle_mod):
    """Measured -> in-process -> disk; a corrupted table is detected and rewritten
    (test_autotune_n54.cpp:273-281, test_cache_invalidation.cpp:240-312)."""
    monkeypatch.setenv("SUNNY_GENEIG_CACHE_DIR", str(tmp_path))
    sbg.tuning_forget_in_process()
    n = 24
    s1 = sbg.Solver(n, tuning="autotune")
    assert s1.was_autotuned and s1.autotune_sweep_ran and s1.cache_layer_used == "measured"
    path = sbg.tuning_table_path(0)
    assert os.path.exists(path)
    s2 = sbg.Solver(n, tuning="autotune")
    assert s2.cache_layer_used == "in-process" and not s2.autotune_sweep_ran
    sbg.tuning_forget_in_process()
    s3 = sbg.Solver(n, tuning="autotune")
    assert s3.cache_layer_used == "disk"
    # corrupt the first bytes, as the reference's invalidation test does
    data = open(path, "rb").read()
    open(path, "wb").write(b"XXXX" + data[4:])
    sbg.tuning_forget_in_process()
    s4 = sbg.Solver(n, tuning="autotune")
    assert s4.cache_layer_used == "measured" and s4.autotune_sweep_ran
    assert open(path, "rb").read()[:7] == b"SBGTUNE"
    # every schedule gives the same answer to rounding
    H, S = oracle_mod.gen_fixture_pairs(n, 8, 3, "random")
    Wr, Xr, _ = oracle_mod.hegv(H, S, n)
    for s in (s1, s4, sbg.Solver(n, tuning="autotune", cache="none"), sbg.Solver(n)):
        dA, dB = dev(H), dev(S)
        W = torch.empty((8, n), dtype=torch.float64, device="cuda"); X = torch.empty_like(dA)
        info = torch.empty(8, dtype=torch.int32, device="cuda")
        s.launch(dA, dB, W, X, info)
        torch.cuda.synchronize()
        assert Mx.eig_rel(W.cpu().numpy(), Wr).max() < 1e-12


def test_cuda_graph_capture_after_reserve(oracle_mod):
    n = 54
    H, S = oracle_mod.gen_fixture_pairs(n, 16, 6, "random")
    Wr, _, _ = oracle_mod.hegv(H, S, n)
    s = sbg.Solver(n)
    s.reserve(16)
    dA, dB = dev(H), dev(S)
    W = torch.empty((16, n), dtype=torch.float64, device="cuda"); X = torch.empty_like(dA)
    info = torch.empty(16, dtype=torch.int32, device="cuda")
    st = torch.cuda.Stream()
    with torch.cuda.stream(st):
        s.launch(dA, dB, W, X, info, stream=st)      # warm-up outside capture
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g, stream=st):
        s.launch(dA, dB, W, X, info, stream=st)
    W.zero_()
    g.replay()
    torch.cuda.synchronize()
    assert Mx.eig_rel(W.cpu().numpy(), Wr).max() < 1e-12
    del g
