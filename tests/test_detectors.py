"""Host side of the modal detectors (no GPU): the per-frequency powers that
measurements() forms from one host copy equal Monitor.power()'s, value for
value, on x- and y-normal planes."""

import numpy as np


class _Solver:
    pass


def test_powers_from_one_copy_equal_power():
    from warp_fdtd_b200.detectors import Monitor

    rng = np.random.default_rng(1)
    for axis, shape in ((0, (1, 30, 20)), (1, (25, 1, 20))):
        m = Monitor.__new__(Monitor)  # host fields only: no device accumulator
        m.axis, m.shape, m.name = axis, shape, "mon"
        m.area_numpy = rng.random(shape)
        s = _Solver()
        K = 3
        c64 = lambda: (rng.standard_normal((K, 3) + shape)  # noqa: E731
                       + 1j * rng.standard_normal((K, 3) + shape)).astype(np.complex64)
        s.data = {"mon/_mode_E": c64(), "mon/_mode_H": c64()}
        raw = rng.standard_normal((K, 6, int(np.prod(shape)), 2))
        ph_all = raw.view(np.complex128)[..., 0].reshape((K, 6) + shape)
        ph_old = (raw[..., 0] + 1j * raw[..., 1]).reshape((K, 6) + shape)
        fast = m.powers(s, ph_all)
        slow = [m.power(s, k, ph_old[k]) for k in range(K)]
        assert fast == slow
        assert all(v > 0 for v in fast)
