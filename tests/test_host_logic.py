"""Host-side logic that needs no GPU: sharding over ranks (gloo, world size 2),
autotuner cache, workload generators, roofline counts, solver argument errors."""
import os
import socket
from types import SimpleNamespace

import numpy as np
import pytest
import torch
import torch.multiprocessing as mp


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _shard(rank):
    g = torch.Generator().manual_seed(100 + rank)
    return torch.randn(3 + 2 * rank, 16, generator=g, dtype=torch.float64)  # unequal shards: 3 and 5 rows


def _rank_main(rank, world, port, out_dir):
    import torch.distributed as dist
    from inc_b200.sharding import gather_rows, max_over_ranks, partition_rows
    from inc_b200.workloads import burgers_batched_config
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    cfg = burgers_batched_config(rows=37, steps=5)
    work = [int(n) * cfg["steps"] for n in cfg["n"]]
    parts = partition_rows(work, world)
    mine = parts[rank]
    # each rank "computes" its rows: a row-dependent value standing in for the solver output
    local = torch.tensor([[float(i), float(cfg["n"][i])] for i in mine], dtype=torch.float64)
    full = gather_rows(local, parts, rank, world)
    t = max_over_ranks(1.0 + rank)
    # data-parallel corrector gradients: each rank's mean loss over its own shard, averaged
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.sharding import allreduce_mean_, average_gradients_
    torch.manual_seed(0)
    net = PeriodicCNN1D(channels=4).double()
    x = _shard(rank)
    net(x).square().mean().backward()
    if rank == 1:  # a parameter that took no part in this rank's loss has no gradient here
        net.convs[0].bias.grad = None
    average_gradients_(net.parameters(), local_rows=x.shape[0])
    grads = [p.grad.clone() for p in net.parameters()]
    try:
        allreduce_mean_([grads[0], None])
        none_rejected = False
    except ValueError:
        none_rejected = True
    pair = [torch.full((2,), float(rank + 1), dtype=torch.float64)]
    allreduce_mean_(pair)
    torch.save({"full": full, "t": t, "parts": parts, "grads": grads, "none_rejected": none_rejected,
                "pair": pair[0], "bias_grad0": net.convs[0].bias.grad is not None}, os.path.join(out_dir, f"rank{rank}.pt"))
    dist.barrier()
    dist.destroy_process_group()


def test_sharding_gloo_world2(tmp_path):
    world = 2
    mp.spawn(_rank_main, args=(world, _free_port(), str(tmp_path)), nprocs=world, join=True)
    from inc_b200.workloads import burgers_batched_config
    cfg = burgers_batched_config(rows=37, steps=5)
    res = [torch.load(tmp_path / f"rank{r}.pt") for r in range(world)]
    for r in res:
        assert r["t"] == 2.0                                    # max over ranks
        assert torch.equal(r["full"][:, 0], torch.arange(37, dtype=torch.float64))
        assert np.array_equal(r["full"][:, 1].numpy(), cfg["n"].astype(np.float64))
    p = res[0]["parts"]
    assert sorted(p[0] + p[1]) == list(range(37)) and res[1]["parts"] == p
    loads = [sum(int(cfg["n"][i]) for i in q) for q in p]
    assert max(loads) - min(loads) <= 512                      # within one largest row
    # row-weighted shard gradients == the gradient of the mean loss over the whole batch,
    # also where one rank had no gradient for a parameter: that rank's share counts as zero
    from inc_b200.correctors import PeriodicCNN1D
    torch.manual_seed(0)
    net = PeriodicCNN1D(channels=4).double()
    net(torch.cat([_shard(r) for r in range(world)])).square().mean().backward()
    torch.manual_seed(0)
    net0 = PeriodicCNN1D(channels=4).double()
    net0(_shard(0)).square().mean().backward()
    rows0, rows = _shard(0).shape[0], sum(_shard(r).shape[0] for r in range(world))
    for r in res:
        assert r["none_rejected"] and r["bias_grad0"]
        assert torch.equal(r["pair"], torch.full((2,), 1.5, dtype=torch.float64))
        for i, (g, p) in enumerate(zip(r["grads"], net.parameters())):
            want = p.grad if i != 1 else net0.convs[0].bias.grad * rows0 / rows
            torch.testing.assert_close(g, want, rtol=1e-12, atol=1e-14)


def test_partition_properties():
    from inc_b200.sharding import contiguous_rows, partition_rows
    w = [5, 1, 1, 1, 9, 3, 3, 2]
    parts = partition_rows(w, 3)
    assert sorted(sum(parts, [])) == list(range(8))
    assert partition_rows(w, 3) == parts
    assert [len(contiguous_rows(10, r, 3)) for r in range(3)] == [4, 3, 3]
    assert list(contiguous_rows(10, 2, 3)) == [7, 8, 9]
    with pytest.raises(ValueError):
        partition_rows(w, 0)


def test_autotune_cache_roundtrip(tmp_path, monkeypatch):
    from inc_b200 import autotune
    monkeypatch.setenv("INC_B200_AUTOTUNE_CACHE", str(tmp_path / "at.json"))
    monkeypatch.setattr(autotune, "_cache", None)
    assert autotune.bucket(1000) == 1024 and autotune.bucket(1024) == 1024 and autotune.bucket(1) == 1
    assert autotune.ks_candidates(256) == [16, 32, 64]
    assert autotune.ks_candidates(16) == [4]
    assert autotune.burgers_candidates(512) == [1, 2, 16]
    assert autotune.burgers_candidates(128) == [1, 2, 4, 8, 16]
    assert autotune.burgers_candidates(32) == [4, 8]
    k = autotune.key("ks", 256, 1000, "ETRK2", None)
    assert k.endswith("|ks|n256|b1024|ETRK2")
    autotune._load()[k] = {"threads_per_pair": 16}
    autotune._save()
    monkeypatch.setattr(autotune, "_cache", None)
    assert autotune.best_ks(256, 700, "ETRK2", None) == 16       # same bucket
    assert autotune.best_ks(256, 5000, "ETRK2", None) == 0       # untuned: library default


def test_workloads_are_seeded_and_shaped():
    from inc_b200.workloads import (burgers_batched_config, burgers_plain_config, ks_diff_config,
                                    ks_plain_config)
    a, b = ks_plain_config(B=8), ks_plain_config(B=8)
    assert np.array_equal(a["u0"], b["u0"]) and np.array_equal(a["s"], b["s"])
    assert a["u0"].shape == (8, 256) and abs(a["s"].std() - 0.01) < 0.003
    c = burgers_plain_config()
    assert c["u0"].shape == (32, 128) and np.abs(c["u0"]).max() <= 2.5
    r = burgers_batched_config(rows=64, steps=3)
    assert set(np.unique(r["n"])) <= {64, 128, 256, 512} and r["nu"].min() >= 1e-3 and r["nu"].max() <= 5e-2
    for u, n, dt, dx, nu in zip(r["u0"], r["n"], r["dt"], r["dx"], r["nu"]):
        assert u.shape == (n,) and dt <= 0.4 * dx / np.abs(u).max() + 1e-15 and dt <= 0.4 * dx * dx / nu + 1e-15
    assert ks_diff_config(B=4)["u0"].shape == (4, 512)


def test_roofline_counts():
    from inc_b200.roofline import BURGERS_FLOPS, ks_flops_per_cell_step, ks_impl_flops_per_cell_step
    assert BURGERS_FLOPS["euler"] == 167 and BURGERS_FLOPS["ssprk3"] == 503
    assert ks_flops_per_cell_step(256) == 490 and ks_flops_per_cell_step(512) == 540  # frozen reference counts
    assert ks_impl_flops_per_cell_step(256) == 184
    assert ks_impl_flops_per_cell_step(256, "ETD1") == 2 * (5 * 8 + 8)


def test_solver_errors_without_gpu():
    from inc_b200.solvers import BurgersSolverTorch, KSSolverTorch
    base = dict(resolution=64, dt=0.01, x=None, adaptive_CFL=None, L=6.28, nu=0.01, device="cpu",
                equation_type="viscosity", batch_size=2)
    with pytest.raises(ValueError, match="Convection scheme not recognized"):
        BurgersSolverTorch(SimpleNamespace(convection_term="upwind", **base))
    with pytest.raises(ValueError):
        BurgersSolverTorch(SimpleNamespace(convection_term="WENO", time_scheme="rk4", **base))
    with pytest.raises(KeyError):
        KSSolverTorch(SimpleNamespace(resolution=64, dt=0.1, device="cpu", domain_size=torch.ones(2),
                                      alpha=torch.zeros(2), time_scheme="RK4"))
    s = BurgersSolverTorch(SimpleNamespace(convection_term="WENO", **base))
    with pytest.raises(ValueError, match="CUDA"):
        s.step(torch.zeros(2, 64))                                  # no CPU path


def test_cnn_weight_packing_layout():
    """pack_cnn_weights: w1[co][k], b1, w2[ci][co][k], b2, w3[ci][co][k], b3, w4[ci][k], b4 (CPU)."""
    import torch
    from inc_b200 import _native as nat
    from inc_b200.correctors import PeriodicCNN1D
    from inc_b200.fused import pack_cnn_weights
    torch.manual_seed(0)
    net = PeriodicCNN1D()
    w = pack_cnn_weights(net)
    assert w.numel() == nat.INC_CNN_WEIGHT_FLOATS == 10657
    c = net.convs
    C, K = 32, 5
    o_b1 = C * K
    o_w2 = o_b1 + C
    o_b2 = o_w2 + C * C * K
    o_w3 = o_b2 + C
    o_b3 = o_w3 + C * C * K
    o_w4 = o_b3 + C
    o_b4 = o_w4 + C * K
    assert torch.equal(w[:o_b1].view(C, K), c[0].weight[:, 0, :])
    assert torch.equal(w[o_b1:o_w2], c[0].bias)
    for ci, co, k in [(0, 0, 0), (3, 17, 4), (31, 5, 2), (12, 31, 1)]:
        assert w[o_w2 + (ci * C + co) * K + k] == c[1].weight[co, ci, k]
        assert w[o_w3 + (ci * C + co) * K + k] == c[2].weight[co, ci, k]
    assert torch.equal(w[o_b2:o_w3], c[1].bias) and torch.equal(w[o_b3:o_w4], c[2].bias)
    assert torch.equal(w[o_w4:o_b4].view(C, K), c[3].weight[0])
    assert w[o_b4] == c[3].bias[0]
    bad = PeriodicCNN1D(channels=16)
    try:
        pack_cnn_weights(bad)
        raise AssertionError("expected ValueError")
    except ValueError:
        pass


def test_spectral_conv_dispatch_on_cpu():
    """CPU tensors never reach inc_spectral_conv1d; the layer is the torch FFT formulation there."""
    import torch
    from inc_b200.correctors import SpectralConv1d, spectral_conv1d_torch, spectral_conv_supported
    torch.manual_seed(0)
    layer = SpectralConv1d(8, 8, 4)
    x = torch.randn(3, 8, 32)
    w_re, w_im = layer.weights_re_im(x.dtype)
    assert not spectral_conv_supported(x, w_re, w_im, 4)
    torch.testing.assert_close(layer(x), spectral_conv1d_torch(x, w_re, w_im, 4), rtol=0, atol=0)
