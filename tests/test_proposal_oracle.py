"""The CPU oracle of the proposal network (oracle/proposal_oracle.py) is
itself checked here: analytic gradients against central finite differences,
rotation equivariance, and the flat parameter layout of the binding.  The GPU
kernels are then checked against this oracle in tests/test_gpu_proposal.py."""
import numpy as np

from oracle import proposal_oracle as po
from rome_b200.proposal import dict_to_flat, expand_proposals, flat_to_dict, param_offsets, posterior_targets


def _setup(seed=0, n_r=5, n_theta=6, ch=(3, 4), K=3, n=3):
    rng = np.random.default_rng(seed)
    params = {name: rng.normal(0, 0.3, shape) for name, shape in po.param_shapes(n_r, n_theta, ch, K)}
    x = rng.normal(size=(n, 2, n_r, n_theta))
    t = rng.dirichlet(np.ones(K * n_theta), size=n)
    return params, x, t


def test_oracle_gradients_match_finite_differences():
    params, x, t = _setup()
    loss, g, _ = po.loss_and_grads(params, x, t)
    rng = np.random.default_rng(1)
    for name, arr in params.items():
        for _ in range(4):
            idx = tuple(rng.integers(0, s) for s in arr.shape)
            old = arr[idx]
            h = 1e-6
            arr[idx] = old + h
            lp = po.loss_and_grads(params, x, t)[0]
            arr[idx] = old - h
            lm = po.loss_and_grads(params, x, t)[0]
            arr[idx] = old
            fd = (lp - lm) / (2 * h)
            assert abs(fd - g[name][idx]) <= 1e-6 + 1e-5 * abs(fd), (name, idx, fd, g[name][idx])


def test_rotation_equivariance():
    """A particle rotated by psi sees its magnitude at angle theta + psi, i.e.
    the input rolled by -psi along theta; the outputs then roll by +psi."""
    params, x, t = _setup(n=2)
    z0, _ = po.forward(params, x)
    z1, _ = po.forward(params, np.roll(x, -2, axis=3))
    K, A = 3, 6
    np.testing.assert_allclose(z1.reshape(2, K, A), np.roll(z0.reshape(2, K, A), 2, axis=2), rtol=1e-10, atol=1e-12)


def test_flat_layout_round_trip():
    n_r, n_theta, ch, K = 5, 6, (3, 4), 3
    params, _, _ = _setup(n_r=n_r, n_theta=n_theta, ch=ch, K=K)
    flat = dict_to_flat(params, n_r, n_theta, ch, K)
    assert flat.size == param_offsets(n_r, n_theta, ch, K)[-1][2]
    for _, _, off in param_offsets(n_r, n_theta, ch, K):
        assert off % 4 == 0
    back = flat_to_dict(flat, n_r, n_theta, ch, K)
    for k in params:
        np.testing.assert_allclose(back[k], params[k], rtol=1e-6, atol=1e-7)


def test_targets_and_expansion():
    K, npsi = 3, 8
    marg = np.zeros((2, K * npsi))
    marg[0, 1 * npsi + 2] = 0.7   # class 1, psi 2
    marg[0, 1 * npsi + 6] = 0.3   # class 1, psi 6 = psi 2 + 180
    marg[1, 2 * npsi + 0] = 1.0
    t = posterior_targets(marg, K, npsi)
    assert t.shape == (2, K * npsi // 2)
    assert t[0, 1 * 4 + 2] == 1.0 and t[1, 2 * 4 + 0] == 1.0
    j = expand_proposals(np.array([[1 * 4 + 2, 0]]), npsi)
    assert j.tolist() == [[0, 4, 1 * 8 + 2, 1 * 8 + 6]]
