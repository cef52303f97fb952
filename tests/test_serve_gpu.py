"""The SCF server (pspw_server_*): independent ChebySCF jobs run with
continuous batching on one GPU give the same results as each job run alone;
admission respects the HBM budget; a failing job does not stop the others.

Jobs are small synthetic clusters of up to four species (pspw.serve), so
the whole file runs in seconds.  Bar: each job's total energy and
eigenvalues in the mix equal the job run alone through
pspw_system_cheby_scf_with with the same controls (the jobs share no data,
so the arithmetic is the same; the test asserts equality to 1e-12 Ha).
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")
if not torch.cuda.is_available():  # pragma: no cover
    pytest.skip("needs a CUDA device", allow_module_level=True)

from pspw import PREC_F32, PREC_F64, serve  # noqa: E402
from pspw.system import System  # noqa: E402

CONTROLS = dict(pulay_beta=0.3, mixdim=6, max_scf_iter=60)


@pytest.fixture(scope="module")
def jobs(tmp_path_factory):
    rng = np.random.default_rng(44)
    sp = serve.species_set(rng)
    out = []
    for k, nat in enumerate((2, 3, 4, 5, 3)):
        d = tmp_path_factory.mktemp(f"job{k}")
        out.append(serve.cluster_job(rng, str(d), sp, natoms=nat, ecut_ha=12.0, box=10.5))
    return out


def _alone(job, prec):
    S = System(job["dir"])
    nat = job["natoms"]
    r = S.cheby_scf(filter_prec=prec, conv=1e-6 * nat, **CONTROLS)
    S.close()
    return r


@pytest.mark.parametrize("prec", [PREC_F64, PREC_F32])
def test_jobs_in_the_mix_equal_jobs_alone(jobs, prec):
    alone = [_alone(j, prec) for j in jobs]
    srv = serve.Server(slots=3, filter_prec=prec, conv_per_atom=1e-6, **CONTROLS)
    ids = [srv.submit(j["dir"]) for j in jobs]
    res = [srv.wait(i, neig=len(a["eig"])) for i, a in zip(ids, alone)]
    srv.close()
    for j, a, r in zip(jobs, alone, res):
        assert r["status"] == 0, r["error"]
        assert r["natoms"] == j["natoms"]
        assert r["iterations"] == a["iterations"]
        assert r["converged"] == int(a["converged"])
        assert abs(r["etot"] - a["energies"]["ETOT"]) <= 1e-12
        assert np.abs(r["eig"] - a["eig"]).max() <= 1e-12
    # several jobs were on the device at the same time
    spans = sorted((r["t_admit"], r["t_done"]) for r in res)
    assert any(spans[k + 1][0] < spans[k][1] for k in range(len(spans) - 1))


def test_budget_admits_one_job_at_a_time(jobs):
    srv = serve.Server(slots=3, hbm_budget_bytes=1.0, conv_per_atom=1e-6, **CONTROLS)
    ids = [srv.submit(j["dir"]) for j in jobs[:3]]
    res = [srv.wait(i) for i in ids]
    srv.close()
    spans = sorted((r["t_admit"], r["t_done"]) for r in res)
    for k in range(len(spans) - 1):
        assert spans[k + 1][0] >= spans[k][1]  # no overlap: each exceeds the budget alone
    assert all(r["status"] == 0 and r["footprint_bytes"] > 1.0 for r in res)


def test_failing_job_does_not_stop_the_server(jobs, tmp_path):
    srv = serve.Server(slots=2, conv_per_atom=1e-6, **CONTROLS)
    bad = srv.submit(str(tmp_path / "no_such_job"))
    good = srv.submit(jobs[0]["dir"])
    rb, rg = srv.wait(bad), srv.wait(good)
    srv.close()
    assert rb["status"] != 0 and rb["error"]
    assert rg["status"] == 0 and rg["iterations"] > 0, rg["error"]
