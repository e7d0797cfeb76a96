"""GPU fault injection on the host side: a non-physical value planted in
the initial data makes the step hit the reference's STOP sites; the kernels
report them as the same status bits the oracle raises on the same state,
the call returns CUEVA_ERR_PHYSICS instead of stopping, and the context
stays usable once the caller restores a good state and clears the bits.
Nothing here faults the GPU: the kernels only see unusual numbers."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

PRIMS = ["rho", "p", "vx", "vy", "vz", "psi", "phi", "Ex", "Ey", "Ez", "Bx", "By", "Bz", "q"]


def _plant(pr, fault):
    j, i = 16, 32
    if fault == "negative_pressure":
        pr["p"][j, i] = -0.5
    elif fault == "superluminal":
        pr["vx"][j, i] = 0.9
        pr["vy"][j, i] = 0.9
    elif fault == "nan_density":
        pr["rho"][j, i] = np.nan


@pytest.mark.parametrize("fault", ["negative_pressure", "superluminal", "nan_density"])
@pytest.mark.parametrize("solver,c2p", [(7, 1), (5, 0), (6, 1)])
def test_planted_fault_reported_like_the_oracle(oracle_mod, solver, c2p, fault):
    from cueva import Cueva, CuevaError
    kw = dict(order=2, flux_solver=solver, rec_mp=0, c2p=c2p, sigma=1e3)
    oracle_mod.set_libm_seed(0)
    g = Cueva(64, 32, **kw)
    o = oracle_mod.Oracle(64, 32, **kw)
    g.kh_init(v0=0.5, a=0.05)
    pr = g.prims()
    _plant(pr, fault)
    for n in PRIMS:
        g.set_interior(n, pr[n])
    o.set_prims(pr)
    g.upload()
    g.step(1)
    st_o = o.step(1)
    if st_o:
        with pytest.raises(CuevaError) as e:
            g.download()
        assert e.value.code == 4
    else:
        g.download()
    assert g.status() == st_o, (g.status(), st_o)
    # the context stays usable: restore a good state, clear, step
    g.kh_init(v0=0.5, a=0.05)
    g.upload()
    g.clear_status()
    g.step(2)
    g.download()
    assert g.status() == 0
    assert all(np.all(np.isfinite(g.interior(n))) for n in PRIMS)
    g.close()
