"""Host side of the SCF serving workload (no GPU): the synthetic cluster
jobs are valid inputs in the reference's formats, with the stated sizes,
and the Poisson schedule is seeded."""
import numpy as np

from pspw import serve
from pspw.system import System


def test_smooth_grid():
    assert serve.smooth_grid(23.2) == 24
    assert serve.smooth_grid(49) == 50
    assert serve.smooth_grid(61) == 64
    assert serve.smooth_grid(70) == 72
    assert serve.smooth_grid(109.03) == 120  # 24 bohr at 25 Ha
    assert serve.smooth_grid(300) == 128  # clipped
    for n in range(24, 129):
        m = serve.smooth_grid(n)
        k = m
        for p in (2, 3, 5):
            while k % p == 0:
                k //= p
        assert k == 1 and m >= n


def test_cluster_jobs_load_host_only(tmp_path):
    rng = np.random.default_rng(3)
    sp = serve.species_set(rng)
    assert all(1.0 <= d <= 4.0 and 0.8 <= w <= 1.6 for d, w in sp)
    for k in range(4):
        j = serve.cluster_job(rng, str(tmp_path / f"j{k}"), sp, natoms_range=(2, 20))
        S = System(j["dir"], device=-1)  # readers, basis and occupations only
        nat = j["natoms"]
        assert S.dims["nr"] == (j["grid"],) * 3
        assert S.dims["nx"] == int(np.ceil(0.6 * 4 * nat)) + 8 == j["nx"]
        assert abs(S.scalars["nel"] - 4 * nat) < 1e-12
        assert S.dims["nsp"] == len(set(j["species"]))
        S.close()


def test_cluster_geometry(tmp_path):
    rng = np.random.default_rng(5)
    sp = serve.species_set(rng)
    j = serve.cluster_job(rng, str(tmp_path / "g"), sp, natoms=30, box=16.0)
    S = System(j["dir"], device=-1)
    tau = S.array("tau")  # (3, nax, nsp), bohr
    na = [int(x) for x in np.bincount(j["species"], minlength=4) if x]
    pos = np.concatenate([tau[:, :n, s].T for s, n in enumerate(na)])
    S.close()
    assert len(pos) == 30
    d = np.linalg.norm(pos[:, None] - pos[None], axis=-1) + np.eye(30) * 1e9
    assert d.min() >= 2.2 - 1e-9
    assert pos.min() >= 3.0 - 1e-9 and pos.max() <= 13.0 + 1e-9  # 6 bohr of vacuum


def test_poisson_schedule_is_seeded():
    a = serve.poisson_arrivals(np.random.default_rng(9), 5.0, 1000)
    b = serve.poisson_arrivals(np.random.default_rng(9), 5.0, 1000)
    assert np.array_equal(a, b) and np.all(np.diff(a) > 0)
    assert abs(1000 / a[-1] - 5.0) < 0.5
