"""Device-side GET_MODEL of the tori (cumc_model_torus) against the host
generators (problems.torus, problems.torus_cyl) they mirror: the states after
initial_update agree to round-off of the power and sine functions (the
device's pow/sin may differ from the host library's by an ulp), for FP64 and
the mixed form; a grid that is not spherical is refused."""
import numpy as np
import pytest

from cumpic_b200 import _native as N
from cumpic_b200 import problems as P

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative to each array's largest magnitude


def _state(prob, device, precision=N.FP64):
    from cumpic_b200.solver import CUMC3D
    prob.precision = precision
    s = CUMC3D(prob)
    if device:
        s.generate_model()
    else:
        s.upload()
    s.initial_update()
    return s, s.download()


TORI = [("spherical", P.torus, (48, 32, 16)), ("cylindrical", P.torus_cyl, (40, 8, 40))]


@pytest.mark.parametrize("name,make,args", TORI, ids=[t[0] for t in TORI])
@pytest.mark.parametrize("precision", [N.FP64, N.MIXED])
def test_device_torus_matches_host_generator(name, make, args, precision):
    _, host = _state(make(*args), False, precision)
    sim, dev = _state(make(*args, host_arrays=False), True, precision)
    for k in host:
        scale = np.max(np.abs(host[k]))
        assert np.max(np.abs(dev[k] - host[k])) <= TOL * scale, k
    # the noise and the normalised field are present, and the run proceeds
    assert np.std(dev["prim"][3:-3, 3:-3, 3:-3, 0]) > 0 and np.max(np.abs(dev["prim"][..., 5])) > 0
    assert np.min(dev["prim"][3:-3, 3:-3, 3:-3, 0]) > 0
    for _ in range(3):
        sim.step()
    assert np.all(np.isfinite(sim.download()["cons"][3:-3, 3:-3, 3:-3]))


def test_model_needs_a_curvilinear_grid():
    from cumpic_b200.solver import CUMC3D
    prob = P.orszag_tang(8)
    prob.model_params = P.torus(8, 8, 4).model_params
    s = CUMC3D(prob)
    with pytest.raises(N.CumcError) as e:
        s.generate_model()
    assert e.value.code == N.CUMC_ERR_CONFIG
