"""The learned face-flux correction: tensor-core forward and backward kernels
against the CPU FP64 restatement (oracle/nn_oracle.py, which rounds to BF16 at
the same points), training, and the corrected solver (conservative, identical to
the plain solver when the network outputs zero, sensor fallback counted)."""
from __future__ import annotations

import numpy as np
import pytest
import torch

from dev_field_efvm_b200 import abi, cases
from oracle import nn_oracle

pytestmark = pytest.mark.gpu


def random_states(batch, n, seed):
    rng = np.random.default_rng(seed)
    y, x = np.meshgrid(np.arange(n) / n, np.arange(n) / n, indexing="ij")
    out = np.zeros((batch, 4, n, n))
    for b in range(batch):
        ph = rng.uniform(0, 2 * np.pi, 4)
        rho = 1.0 + 0.2 * np.sin(2 * np.pi * x + ph[0]) * np.cos(2 * np.pi * y + ph[1])
        u = 0.5 * np.sin(2 * np.pi * y + ph[2])
        v = 0.5 * np.cos(2 * np.pi * x + ph[3])
        p = 1.0 + 0.1 * np.cos(2 * np.pi * (x + y) + ph[0])
        out[b] = np.stack([rho, rho * u, rho * v, p / 0.4 + 0.5 * rho * (u * u + v * v)])
    return out


def trained_like_params(net, seed):
    """Parameters with an output layer large enough that the corrections matter."""
    p = net.params().astype(np.float64)
    rng = np.random.default_rng(seed)
    p[nn_oracle.P_W3:nn_oracle.P_B1] = rng.normal(0, 0.3, nn_oracle.NOUT * nn_oracle.H)
    p[nn_oracle.P_B1:nn_oracle.P_B3] = rng.normal(0, 0.1, 2 * nn_oracle.H)
    p[nn_oracle.P_B3:] = rng.normal(0, 0.1, nn_oracle.NOUT)
    return p.astype(np.float32)


def test_forward_matches_cpu():
    from dev_field_efvm_b200.device import FluxNet

    net = FluxNet(out_scale=1e-2, seed=3)
    p = trained_like_params(net, 1)
    net.set_params(p)
    s = random_states(2, 16, 0)
    st = torch.tensor(s, device="cuda")
    corr = torch.zeros((2, 2, 4, 16, 16), dtype=torch.float32, device="cuda")
    net.forward(st, corr)
    ref, _ = nn_oracle.forward(p.astype(np.float64), s, 1e-2)
    got = corr.cpu().numpy().astype(np.float64)
    err = np.max(np.abs(got - ref)) / np.max(np.abs(ref))
    assert err < 2e-3, err


def test_loss_and_gradient_match_cpu_fp64():
    """The gradient check: every parameter block of the GPU gradient against the
    CPU FP64 one (relative L2 error of each block)."""
    from dev_field_efvm_b200.device import FluxNet

    net = FluxNet(out_scale=1e-2, seed=5)
    p = trained_like_params(net, 2)
    net.set_params(p)
    s = random_states(3, 16, 1)
    rng = np.random.default_rng(9)
    resid = rng.normal(0, 1e-2, s.shape)
    dx = dy = 10.0 / 16
    w = [1.0, 2.0, 2.0, 0.5]
    grad = torch.zeros(net.P, dtype=torch.float32, device="cuda")
    loss = net.loss_grad(torch.tensor(s, device="cuda"), torch.tensor(resid, device="cuda"), dx, dy, w, grad)
    ref_loss, ref_grad, _ = nn_oracle.loss_grad(p.astype(np.float64), s, resid, dx, dy, w, 1e-2)
    assert abs(loss - ref_loss) <= 1e-5 * ref_loss
    g = grad.cpu().numpy().astype(np.float64)
    blocks = {"W1": (nn_oracle.P_W1, nn_oracle.P_W2), "W2": (nn_oracle.P_W2, nn_oracle.P_W3),
              "W3": (nn_oracle.P_W3, nn_oracle.P_B1), "b1": (nn_oracle.P_B1, nn_oracle.P_B2),
              "b2": (nn_oracle.P_B2, nn_oracle.P_B3), "b3": (nn_oracle.P_B3, nn_oracle.P_COUNT)}
    full = np.linalg.norm(ref_grad)
    for name, (a, b) in blocks.items():
        diff = np.linalg.norm(g[a:b] - ref_grad[a:b])
        if name == "b3":
            # a constant flux has no divergence: this gradient is a telescoping sum
            # of cancelling terms, zero up to round-off; judge it against the whole
            assert diff < 1e-4 * full, (name, diff, full)
            continue
        rel = diff / max(np.linalg.norm(ref_grad[a:b]), 1e-30)
        assert rel < 2e-3, (name, rel)


def test_adam_steps_reduce_the_loss():
    from dev_field_efvm_b200.device import FluxNet

    net = FluxNet(out_scale=1e-2, seed=7)
    s = torch.tensor(random_states(4, 16, 2), device="cuda")
    # a residual the network can represent: the divergence of a fixed smooth flux field
    rng = np.random.default_rng(3)
    target = rng.normal(0, 1.0, (4, 2, 4, 16, 16)) * 1e-2
    dx = dy = 10.0 / 16
    cx, cy = target[:, 0], target[:, 1]
    resid = -((np.roll(cx, -1, axis=3) - cx) / dx + (np.roll(cy, -1, axis=2) - cy) / dy)
    r = torch.tensor(resid, device="cuda")
    first = net.loss_grad(s, r, dx, dy, [1, 1, 1, 1])
    for _ in range(200):
        net.loss_grad(s, r, dx, dy, [1, 1, 1, 1])
        net.adam(3e-3)
    last = net.loss_grad(s, r, dx, dy, [1, 1, 1, 1])
    assert last < 0.8 * first, (first, last)


def _vortex_pair(net, sensor=0.0, seam=abi.SEAM_REFERENCE):
    from dev_field_efvm_b200.device import Context

    grid, params, u, ex = cases.vortex_case(64, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4, seam=seam)
    plain, corrected = Context(grid, params), Context(grid, params)
    plain.upload(u)
    corrected.upload(u)
    corrected.set_flux_correction(net, sensor)
    return plain, corrected


def test_zero_network_leaves_the_solver_unchanged():
    from dev_field_efvm_b200.device import FluxNet

    net = FluxNet(out_scale=1e-2, seed=1)
    net.set_params(np.zeros(net.P, dtype=np.float32))
    plain, corrected = _vortex_pair(net)
    plain.step(10)
    corrected.step(10)
    a, b = plain.download(), corrected.download()
    assert np.max(np.abs(a - b)) <= 1e-12 * np.max(np.abs(a))
    faces, fallbacks = corrected.correction_stats()
    assert faces == 10 * 3 * 2 * 64 * 64 and fallbacks == 0


def test_corrected_solver_is_conservative_and_differs():
    from dev_field_efvm_b200.device import FluxNet

    net = FluxNet(out_scale=1e-3, seed=2)
    net.set_params(trained_like_params(net, 4))
    # the conservative seam: the plain method conserves mass to round-off there,
    # and the correction (a difference of face values) must not change that
    plain, corrected = _vortex_pair(net, seam=abi.SEAM_TRUE_PERIODIC)
    m0 = corrected.total_mass()
    plain.step(20)
    corrected.step(20)
    assert abs(plain.total_mass() - m0) <= 1e-13 * m0
    assert abs(corrected.total_mass() - m0) <= 1e-13 * m0
    assert np.max(np.abs(plain.download() - corrected.download())) > 1e-8


def test_sensor_falls_back_at_a_pressure_jump():
    from dev_field_efvm_b200.device import Context, FluxNet

    net = FluxNet(out_scale=1e-3, seed=2)
    net.set_params(trained_like_params(net, 4))
    grid, params, u, ex = cases.vortex_case(64, periodic=True, muscl=True, mean=(1.0, 1.0), cfl=0.4)
    u = u.copy()
    u[:, 20:40, 4] *= 1.5  # a band of cells at 1.5x energy: pressure jumps at its two edges
    c = Context(grid, params)
    c.upload(u)
    c.set_flux_correction(net, sensor=0.2)
    c.step(1)
    faces, fallbacks = c.correction_stats()
    assert faces == 3 * 2 * 64 * 64
    assert fallbacks >= 3 * 2 * 64  # at least the two band edges on every stage
    assert fallbacks < faces // 4
