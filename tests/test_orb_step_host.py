"""donof_orb_step_host (api.OrbStepHost): the host side of one iteration of the
reference's optimiser loop (src/minimization.jl:390-412) against the oracle's
restatement of the same update (oracle/orbital.py: packing of
4 (elag - elag^T), then the AMSGrad family) over several iterations and all
four methods; no GPU."""
import numpy as np
import pytest

import donof_b200 as d
from donof_b200 import _lib
from oracle import gnof as ognof


def reference_steps(method, elags, nbf5, alpha, maxloop):
    beta1, beta2 = (0.6, 0.999) if method == "Demon" else (0.5, 0.9)
    binit = beta1
    nvar = ognof.pack_orbital_gradient(elags[0], nbf5).shape[0]
    m, v, vmax = np.zeros(nvar), np.zeros(nvar), np.zeros(nvar)
    ys = []
    for i, elag in enumerate(elags, start=1):
        g = ognof.pack_orbital_gradient(elag, nbf5)
        if method == "Demon":
            rate = (i - 1.0) / (maxloop - 1.0)
            beta1 = binit * (1.0 - rate) / ((1.0 - binit) + binit * (1.0 - rate))
        m = beta1 * m + (1.0 - beta1) * g
        if method == "ADABelief":
            v = beta2 * v + (1.0 - beta2) * (g - m) ** 2
        elif method == "YOGI":
            v = v - (1.0 - beta2) * np.sign(v - g ** 2) * g ** 2
        else:
            v = beta2 * v + (1.0 - beta2) * g ** 2
        vmax = np.maximum(vmax, v / (1.0 - beta2 ** i))
        ys.append((-alpha * (m / (1.0 - beta1 ** i)) / np.sqrt(vmax + 1e-16), np.max(np.abs(g))))
    return ys


@pytest.mark.parametrize("method", ["ADAM", "ADABelief", "YOGI", "Demon"])
def test_host_step_matches_the_reference_update(method):
    rng = np.random.default_rng(7)
    nbf, nbf5, maxloop = 37, 11, 6
    elags = [np.asfortranarray(rng.standard_normal((nbf, nbf))) for _ in range(maxloop)]
    st = d.OrbStepHost(nbf, nbf5, method, alpha=0.02, maxloop=maxloop)
    for (y0, g0), elag in zip(reference_steps(method, elags, nbf5, 0.02, maxloop), elags):
        y = st.step(elag)
        assert np.allclose(y, y0, rtol=1e-13, atol=1e-16)
        assert st.gmax.value == g0
    st.reset()
    assert np.allclose(st.step(elags[0]), reference_steps(method, elags[:1], nbf5, 0.02, maxloop)[0][0], rtol=1e-13)


def test_host_step_refuses_bad_arguments():
    lib = _lib.load()
    a = np.zeros(10)
    assert lib.donof_orb_step_host(9, 1, 10, 0.01, a.ctypes.data, 3, 2, a.ctypes.data, a.ctypes.data, a.ctypes.data,
                                   a.ctypes.data, a.ctypes.data, None) == _lib.ERR_ARG
    assert lib.donof_orb_step_host(0, 0, 10, 0.01, a.ctypes.data, 3, 2, a.ctypes.data, a.ctypes.data, a.ctypes.data,
                                   a.ctypes.data, a.ctypes.data, None) == _lib.ERR_ARG
    with pytest.raises(ValueError):
        d.OrbStepHost(5, 2).step(np.zeros((4, 4)))
