"""Hand-written adjoints of the FP64 step, checked against central finite
differences: dot-product tests of each vector-Jacobian product, and the full
gradient of a differentiable PM run (loss = MSE between the final CIC density
and a target density from a second seed) with respect to the initial
displacement field, through the checkpointed torch.autograd.Function of
tests/pm_autograd.py."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def T(a):
    return torch.tensor(np.ascontiguousarray(a), dtype=torch.float64, device=DEV)


def lattice(ng, nrow):
    sp = ng / nrow
    i = np.arange(nrow)
    g = [np.broadcast_to(a, (nrow,) * 3).reshape(-1) for a in (i[:, None, None], i[None, :, None], i[None, None, :])]
    return [T((a + 0.5) * sp) for a in g]


def test_adjoint_deposit_dot_product(pmpkg):
    ng, np_ = 32, 5000
    rng = np.random.default_rng(1)
    x = [T(rng.uniform(0, ng, np_)) for _ in range(3)]
    h = [T(rng.standard_normal(np_)) for _ in range(3)]
    dbar = torch.zeros((ng, ng, ng + 2), dtype=torch.float64, device=DEV)
    dbar[:, :, :ng] = torch.randn((ng, ng, ng), dtype=torch.float64, device=DEV)
    plan = pmpkg.Plan(ng, "fp64")
    eps = 1e-6
    dp = plan.deposit(*[a + eps * b for a, b in zip(x, h)], 1.3)
    dm = plan.deposit(*[a - eps * b for a, b in zip(x, h)], 1.3)
    lhs = float(((dp - dm)[:, :, :ng] * dbar[:, :, :ng]).sum()) / (2 * eps)
    xb = [torch.zeros_like(x[0]) for _ in range(3)]
    plan.adjoint_deposit(*x, 1.3, dbar, xb)
    rhs = float(sum((a * b).sum() for a, b in zip(xb, h)))
    assert rhs == pytest.approx(lhs, rel=1e-6)


@pytest.mark.parametrize("kind,order", [("discrete", 2), ("spectral", 4)])
def test_adjoint_force_dot_product(pmpkg, kind, order):
    ng, np_ = 32, 8000
    rng = np.random.default_rng(2)
    x = [T(rng.uniform(2, ng - 2, np_)) for _ in range(3)]
    h = [T(rng.standard_normal(np_)) for _ in range(3)]
    u = [T(rng.standard_normal(np_)) for _ in range(3)]
    plan = pmpkg.Plan(ng, "fp64", kind, order)
    mass, cp, eps = ng ** 3 / np_, 4 * np.pi, 1e-6

    def force(xx):
        f = [torch.zeros_like(x[0]) for _ in range(3)]
        plan.step(*[t.clone() for t in xx], *f, mass, cp, 1.0, 0.0)
        return f

    fp = force([a + eps * b for a, b in zip(x, h)])
    fm = force([a - eps * b for a, b in zip(x, h)])
    lhs = float(sum(((p - m) * w).sum() for p, m, w in zip(fp, fm, u))) / (2 * eps)
    xb = [torch.zeros_like(x[0]) for _ in range(3)]
    plan.adjoint_force(*x, mass, cp, u, 1.0, xb)
    rhs = float(sum((a * b).sum() for a, b in zip(xb, h)))
    assert rhs == pytest.approx(lhs, rel=1e-5)


@pytest.mark.parametrize("ng,nrow,steps,dt,ckpt,ncomp",
                         [(32, 32, 8, 0.01, 3, 64), (128, 128, 32, 0.01, 8, 64)])
def test_run_gradient_matches_finite_differences(pmpkg, O, ng, nrow, steps, dt, ckpt, ncomp):
    """Gradient w.r.t. the initial displacement field, checkpointing every
    `ckpt` steps; the second case is the differentiable-PM configuration
    (128^3 on 128^3, 32 KDK steps at dt = 0.01, checkpoint every 8)."""
    from pm_autograd import loss_fn

    psi0 = O.zeldovich_displacement(nrow, -2.0, seed=11)
    rms = np.sqrt(np.mean(np.sum(psi0 * psi0, axis=0)))
    psi = T((psi0 * (0.5 / rms)).reshape(3, -1)).requires_grad_(True)
    q = lattice(ng, nrow)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    plan = pmpkg.Plan(ng, "fp64", "spectral", 4)
    # target: the final density of a run from a second seed
    tpos, tvel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=12)
    tx = [T(a) for a in tpos]
    tv = [T(a) for a in tvel]
    from pm_autograd import kdk_schedule
    for ck, dd in kdk_schedule(steps, dt)[:-1]:
        plan.step(*tx, *tv, mass, cp, ck, dd)
    target = plan.deposit(*tx, mass)[:, :, :ng].clone()

    loss = loss_fn(psi, q, plan, ng, mass, cp, dt, steps, target, 1.0, ckpt)
    loss.backward()
    g = psi.grad.detach()
    assert torch.isfinite(g).all() and float(g.abs().max()) > 0

    rng = np.random.default_rng(13)
    comps = [(int(rng.integers(3)), int(rng.integers(nrow ** 3))) for _ in range(ncomp)]
    eps = 1e-5
    fd, ad = [], []
    with torch.no_grad():
        for a, p in comps:
            base = psi.detach().clone()
            base[a, p] += eps
            lp = float(loss_fn(base, q, plan, ng, mass, cp, dt, steps, target, 1.0, ckpt))
            base[a, p] -= 2 * eps
            lm = float(loss_fn(base, q, plan, ng, mass, cp, dt, steps, target, 1.0, ckpt))
            fd.append((lp - lm) / (2 * eps))
            ad.append(float(g[a, p]))
    fd, ad = np.array(fd), np.array(ad)
    err = np.linalg.norm(fd - ad) / np.linalg.norm(fd)
    assert err < 1e-4, (err, fd[:5], ad[:5])
