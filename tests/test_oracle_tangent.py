"""The tangent-linear oracle (the FP64 reference gradient of the adjoint
checks) against central differences of the FP64 oracle itself, on CPU.

Its values must equal the double oracle's bit for bit (the same operations
on the value parts), and its derivative parts must match central
differences. A step of 1e-9 keeps the perturbed runs on the base point's
limiter and solver branches on this generic smooth state; the residual is
the differences' round-off.
"""
import numpy as np

from _oracle import Oracle, TangentOracle
from test_gpu_adjoint import _directions, generic_box


def _run(prob, prim, eps, dts):
    o = Oracle(prob, threads=4)
    o.upload(prim, eps)
    o.initial_update()
    for dt in dts:
        o.rungekutta(dt)
    return o.download()


def test_tangent_oracle_values_and_derivatives():
    prob = generic_box(8)
    o = Oracle(prob, threads=4)
    o.upload()
    o.initial_update()
    dts = []
    for _ in range(2):
        dts.append(o.finddt())
        o.rungekutta(dts[-1])
    base = o.download()
    (dp, de), = _directions(prob, 1, 3)
    v, d = TangentOracle(prob, threads=4).run(dp, de, dts)
    for k in v:
        np.testing.assert_array_equal(v[k], base[k])
    h = 1e-9
    a = (slice(3, -3),) * 3
    fp = _run(prob, prob.prim + h * dp, prob.eps + h * de, dts)["cons"][a]
    fm = _run(prob, prob.prim - h * dp, prob.eps - h * de, dts)["cons"][a]
    fd = (fp - fm) / (2 * h)
    tl = d["cons"][a]
    for q in range(8):
        scale = np.max(np.abs(tl[..., q]))
        assert np.max(np.abs(fd[..., q] - tl[..., q])) <= 1e-4 * scale, q
