"""Material gradients of the forward/backward pair (tdbem_md_march_forward /
tdbem_md_march_backward): dJ/dE_d and dJ/drho_d of J = <c_lu, lu> + <c_lt, lt>.

Three checks:
- an exact identity of the discrete model: scaling every domain's E and rho
  by the same factor keeps the wave speeds (so every wave-front window and
  quadrature rule), divides the displacement kernel by the factor and leaves
  the traction kernels alone; with zero prescribed displacements the march's
  displacements then scale by 1/factor and its tractions stay, so
  sum_d (E_d dJ/dE_d + rho_d dJ/drho_d) = -<c_lu, lu>;
- central differences of the whole march (new handle, quadrature and march
  per evaluation, the card material and so dt held fixed) to 1e-5 relative.
  The discrete model is piecewise smooth in the materials (a quadrature point
  crossing a time-step boundary moves its contribution to the neighbouring
  step), so a difference is trusted only when the steps h and 2h agree;
- the load gradient of the pair equals tdbem_md_march_vjp's, and the
  torch.autograd.Function hands the material gradient to a (D, 2) tensor.
"""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _hetero_rod(nstep=24, mats=None, card=None):
    from tdbem import cases
    if mats is None:
        rng = np.random.default_rng(17)
        mats = [cases.Material(rng.uniform(15, 30), 0.25, rng.uniform(15, 25)) for _ in range(5)]
    c = cases.make_case("rod5_grad", 5, 2, mats, 0.6, nstep,
                        [(1.0, (0.6, 0.3, -0.2), cases.heaviside(nstep))], error=1e-14)
    c.card = card if card is not None else mats[0]
    return c


def _cotangents(c, seed=3):
    rng = np.random.default_rng(seed)
    shape = (c.nstep + 1, c.n_elements, 3)
    return rng.normal(size=shape), rng.normal(size=shape)


def _solver(c):
    from tdbem.api import MultiDomainSolver
    s = MultiDomainSolver(c)
    s.assemble()
    return s


def _J(c, c_lu, c_lt):
    s = _solver(c)
    lu, lt, rep = s.march(c.known[0])
    s.close()
    assert rep.steps_solved == c.nstep
    return float(np.sum(c_lu * lu) + np.sum(c_lt * lt))


def test_scaling_identity():
    c = _hetero_rod()
    c_lu, c_lt = _cotangents(c)
    s = _solver(c)
    lu, lt, rep = s.march_forward(c.known[0])
    assert rep.steps_solved == c.nstep
    _, gm, _ = s.march_backward(c_lu, c_lt)
    E = np.array([m.E for m in c.materials])
    rho = np.array([m.rho for m in c.materials])
    lhs = float(np.sum(E * gm[:, 0] + rho * gm[:, 1]))
    rhs = -float(np.sum(c_lu * lu))
    assert np.all(np.isfinite(gm)) and np.any(gm != 0.0)
    assert abs(lhs - rhs) <= 1e-9 * abs(rhs), (lhs, rhs)


def test_central_differences():
    from tdbem import cases
    c = _hetero_rod()
    c_lu, c_lt = _cotangents(c)
    s = _solver(c)
    s.march_forward(c.known[0])
    _, gm, _ = s.march_backward(c_lu, c_lt)
    card = c.materials[0]

    def J_at(d, which, rel):
        mats = list(c.materials)
        m = mats[d]
        mats[d] = cases.Material(m.E * (1 + rel), m.nu, m.rho) if which == 0 else \
            cases.Material(m.E, m.nu, m.rho * (1 + rel))
        return _J(dataclasses.replace(c, materials=mats, card=card), c_lu, c_lt)

    checked = 0
    for d in (0, 2, 4):
        for which in (0, 1):
            theta = c.materials[d].E if which == 0 else c.materials[d].rho
            ad = gm[d, which]
            fd = None
            # largest steps first (least rounding).  A crossing inside +-2h
            # shows as a disagreement of h and 2h of 0.5 to 1e4 (measured);
            # the march's own noise (GMRES to 1e-14) gives up to about 1e-5
            # at h = 1e-8 (E of domain 2 has a crossing within 2e-7, so only
            # the small steps are smooth there)
            for h in (1e-7, 3e-8, 3e-7, 1e-8):
                f1 = (J_at(d, which, h) - J_at(d, which, -h)) / (2 * h * theta)
                f2 = (J_at(d, which, 2 * h) - J_at(d, which, -2 * h)) / (4 * h * theta)
                if abs(f1 - f2) <= 1e-4 * abs(f1):
                    fd = f1
                    break
            assert fd is not None, ("no smooth step found", d, which)
            assert abs(fd - ad) <= 1e-5 * abs(fd), (d, which, fd, ad)
            checked += 1
    assert checked == 6


def test_load_gradient_and_autograd():
    import torch
    from tdbem.api import march_function
    c = _hetero_rod(nstep=16)
    c_lu, c_lt = _cotangents(c, seed=5)
    s = _solver(c)
    s.march_forward(c.known[0])
    gk, gm, _ = s.march_backward(c_lu, c_lt)
    gv, _ = s.march_vjp(c_lu, c_lt)
    assert np.allclose(gk, gv, rtol=0, atol=1e-12 * np.max(np.abs(gv)))
    k = torch.tensor(c.known[0], requires_grad=True)
    mats = torch.tensor([[m.E, m.rho] for m in c.materials], dtype=torch.float64, requires_grad=True)
    lu, lt = march_function().apply(s, k, mats)
    (torch.sum(torch.from_numpy(c_lu) * lu) + torch.sum(torch.from_numpy(c_lt) * lt)).backward()
    assert np.allclose(k.grad.numpy(), gk, rtol=0, atol=1e-12 * np.max(np.abs(gk)))
    assert np.allclose(mats.grad.numpy(), gm, rtol=1e-12, atol=0)


def test_backward_needs_forward():
    from tdbem.api import TdbemError
    c = _hetero_rod(nstep=8)
    s = _solver(c)
    s.march(c.known[0])
    with pytest.raises(TdbemError):
        s.march_backward(*_cotangents(c))


def test_autograd_on_cuda_tensors():
    """CUDA tensors go through the C ABI as device buffers: the same outputs
    and gradients, bit for bit, as the CPU-tensor path."""
    import torch
    from tdbem.api import march_function
    c = _hetero_rod(nstep=16)
    c_lu, c_lt = _cotangents(c, seed=7)
    s = _solver(c)
    f = march_function()
    grads = []
    for dev in ("cpu", "cuda"):
        k = torch.tensor(c.known[0], device=dev, requires_grad=True)
        mats = torch.tensor([[m.E, m.rho] for m in c.materials], dtype=torch.float64, device=dev,
                            requires_grad=True)
        lu, lt = f.apply(s, k, mats)
        J = torch.sum(torch.from_numpy(c_lu).to(dev) * lu) + torch.sum(torch.from_numpy(c_lt).to(dev) * lt)
        J.backward()
        grads.append((lu.detach().cpu().numpy(), k.grad.cpu().numpy(), mats.grad.cpu().numpy()))
    for a, b in zip(grads[0], grads[1]):
        assert np.array_equal(a, b)
