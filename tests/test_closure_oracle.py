"""CPU: the numpy restatement of the closure network (oracle/closure_oracle.py)
that checks the CUDA training kernels: its analytic weight gradients agree
with central finite differences of its own loss."""
import numpy as np

from oracle import closure_oracle as CO


def test_numpy_network_gradients_match_finite_differences():
    rng = np.random.default_rng(0)
    n, D, H, W = 2, 4, 3, 5
    face = np.array([1, 4])
    x = rng.standard_normal((n, 10, D, H, W))
    t = rng.standard_normal((n, 6, D, H, W)) * 0.1
    ws = [rng.standard_normal((6, co, ci, 27)) * 0.2 for ci, co in ((10, 16), (16, 16), (16, 6))]
    loss, grads, _ = CO.net_loss_and_grads(x, t, ws, face, 6)
    for layer, (f, o, c, tap) in enumerate([(1, 3, 7, 13), (4, 0, 15, 26), (1, 5, 2, 0)]):
        h = 1e-5
        wp = [w.copy() for w in ws]
        wm = [w.copy() for w in ws]
        wp[layer][f, o, c, tap] += h
        wm[layer][f, o, c, tap] -= h
        num = (CO.net_loss_and_grads(x, t, wp, face, 6)[0] - CO.net_loss_and_grads(x, t, wm, face, 6)[0]) / (2 * h)
        assert abs(num - grads[layer][f, o, c, tap]) <= 1e-6 * max(1.0, abs(num)), (layer, num)
    # faces without samples get no gradient
    assert not np.any(grads[0][0]) and not np.any(grads[2][5])


def test_bf16_rounding_is_nearest_even():
    v = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 3 * 2 ** -8, -2.5, 0.0], np.float32)
    assert CO.bf16_round(v).tolist() == [1.0, 1.0, 1.0 + 2 ** -6, -2.5, 0.0]
