"""Energy spectrum and trajectory windows vs the reference's own code
(golden vectors from analysis/Plot_KS.py and data/data_loader_1d.py)."""
import numpy as np
import pytest
import torch

from oracle import analysis as oa
from oracle import data as od
from tests.golden_io import load, rel_l2

AZ = load("analysis_data_golden.npz")


@pytest.mark.parametrize("name", ["spec_even", "spec_even2d", "spec_256"])
def test_oracle_spectrum_matches_reference(name):
    e, k = oa.energy_spectrum(AZ[f"{name}.v"])
    assert rel_l2(e, AZ[f"{name}.energy"]) < 1e-6
    assert np.allclose(k, AZ[f"{name}.k"])


def _data():
    d = {k: torch.from_numpy(AZ[f"dl.{k}"]) for k in ("trajectories", "nu", "A", "omega", "phi", "l", "domain_size")}
    d["metadata"] = {"gen_dt": 0.5}
    return d


@pytest.mark.parametrize("case", [str(c) for c in AZ["dl.cases"]])
def test_windows_match_reference_datasets(case):
    from inc_b200.data import TrajectoryWindows
    dt, mstep, gap = AZ[f"dl.{case}.args"]
    kind = "burgers" if case.startswith("bg") else "ks"
    w = TrajectoryWindows(_data(), dt=dt, mstep=int(mstep), starts_gap=int(gap), kind=kind, device="cpu")
    assert len(w) == int(AZ[f"dl.{case}.len"])
    b = w.batch(torch.arange(len(w)))
    assert np.array_equal(b["u_initial"].numpy(), AZ[f"dl.{case}.u_initial"])
    assert np.array_equal(b["u_target"].numpy(), AZ[f"dl.{case}.u_target"])
    if kind == "burgers":
        assert np.allclose(b["t"].numpy(), AZ[f"dl.{case}.t"])
        assert np.array_equal(b["nu"].numpy(), AZ[f"dl.{case}.nu"])
    else:
        assert np.array_equal(b["domain_size"].numpy(), AZ[f"dl.{case}.domain_size"].reshape(-1))
    items = od.windows(AZ["dl.trajectories"], 0.5, dt, int(mstep), int(gap))
    assert np.array_equal(np.stack([it[2] for it in items]), AZ[f"dl.{case}.u_initial"])
    # the loader visits every item once, in batches
    seen = torch.cat([x["u_initial"] for x in w.loader(4, shuffle=True, generator=torch.Generator().manual_seed(0))])
    assert seen.shape[0] == len(w)


def test_windows_reject_non_multiple_dt():
    from inc_b200.data import TrajectoryWindows
    with pytest.raises(ValueError):
        TrajectoryWindows(_data(), dt=0.7, mstep=2, kind="ks", device="cpu")


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["spec_even", "spec_even2d", "spec_256"])
def test_gpu_spectrum_matches_reference(cuda, name):
    from inc_b200.analysis import energy_spectrum
    e, k = energy_spectrum(torch.tensor(AZ[f"{name}.v"], device=cuda))
    assert rel_l2(e.cpu().numpy(), AZ[f"{name}.energy"]) < 1e-5
    assert np.allclose(k.cpu().numpy(), AZ[f"{name}.k"], rtol=1e-6)


@pytest.mark.gpu
@pytest.mark.parametrize("n", [16, 32, 64, 128, 256, 512])
def test_gpu_spectrum_sizes(cuda, n):
    from inc_b200.analysis import energy_spectrum
    rng = np.random.default_rng(n)
    v = rng.standard_normal((3, 5, n)).astype(np.float32)  # 15 rows: a lone row at the end
    e, _ = energy_spectrum(torch.tensor(v, device=cuda))
    assert rel_l2(e.cpu().numpy(), oa.energy_spectrum(v)[0]) < 1e-5


@pytest.mark.gpu
def test_gpu_generated_ks_dataset_windows(cuda):
    from types import SimpleNamespace
    from inc_b200.data import TrajectoryWindows, generate_ks
    from inc_b200.solvers import KSSolverTorch
    from inc_b200.workloads import ks_u0
    from oracle import ks as oks
    B, N, dt = 4, 64, 0.1
    Ls = [40.0, 40.0, 50.0, 64.0]
    ds = torch.tensor(Ls, device=cuda)
    solver = KSSolverTorch(SimpleNamespace(resolution=N, dt=dt, device=cuda, domain_size=ds,
                                           alpha=torch.zeros(B, device=cuda), time_scheme="ETRK2"))
    rng = np.random.default_rng(0)
    u0 = np.stack([ks_u0(rng, 1, N, L)[0] for L in Ls])
    data = generate_ks(solver, torch.tensor(u0, dtype=torch.float32, device=cuda), ds, 12)
    assert data["trajectories"].shape == (B, 13, N) and data["metadata"]["gen_dt"] == pytest.approx(0.2)
    ref = u0
    for k in range(1, 13):
        ref = oks.step(ref, Ls, dt, "ETRK2")
        assert rel_l2(data["trajectories"][:, k].cpu().numpy(), ref) < 1e-5
    w = TrajectoryWindows(data, dt=0.4, mstep=2, starts_gap=1, kind="ks")
    i = torch.arange(len(w), device=cuda)
    b = w.batch(i)
    row, start = i // len(w.starts), w.starts[i % len(w.starts)]
    assert torch.equal(b["u_target"][:, -1], data["trajectories"][row, start + 4])  # 2 windows of 2 frames
    assert torch.equal(b["domain_size"], ds[row])
