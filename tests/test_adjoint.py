"""Hand-written adjoints of the step, checked against central finite
differences: dot-product tests of each FP64 vector-Jacobian product, and the
full gradient of a differentiable PM run (loss = MSE between the final CIC
density and a target density from a second seed) with respect to the initial
displacement field, through the checkpointed torch.autograd.Function of
tests/pm_autograd.py.  The FP32 split-position adjoints are checked against
the FP64 ones (per product and for the whole run) and against the same finite
differences."""
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


# ---------------------------------------------------- FP32 split positions
@pytest.mark.parametrize("ng,kind,order", [(32, "discrete", 2), (64, "spectral", 4)])
def test_adjoint_f32_products_match_f64(pmpkg, ng, kind, order):
    """pm_adjoint_deposit_f32 / pm_adjoint_force_f32 against the FP64
    products at the same positions (FP32 arithmetic: relative L2 < 1e-4)."""
    np_ = 4 * ng ** 3 // 8
    rng = np.random.default_rng(ng)
    x = [T(rng.uniform(0, ng, np_)) for _ in range(3)]
    u = [T(rng.standard_normal(np_)) for _ in range(3)]
    p64, p32 = pmpkg.Plan(ng, "fp64", kind, order), pmpkg.Plan(ng, "fp32", kind, order)
    cell, off = p32.split(*x)
    x = p32.join(cell, off)  # the FP64 side at exactly the FP32 positions
    mass, cp = ng ** 3 / np_, 4 * np.pi
    dbar = torch.zeros((ng, ng, ng + 2), dtype=torch.float64, device=DEV)
    dbar[:, :, :ng] = torch.randn((ng, ng, ng), dtype=torch.float64, device=DEV)

    def rel(a, b):
        a, b = torch.stack(a).double(), torch.stack(b)
        return float((a - b).norm() / b.norm())

    b64 = [torch.zeros_like(x[0]) for _ in range(3)]
    b32 = [torch.zeros(np_, dtype=torch.float32, device=DEV) for _ in range(3)]
    p64.adjoint_deposit(*x, mass, dbar, b64)
    p32.adjoint_deposit_split(cell, off, mass, dbar.float(), b32)
    assert rel(b32, b64) < 1e-5
    b64 = [torch.zeros_like(x[0]) for _ in range(3)]
    b32 = [torch.zeros(np_, dtype=torch.float32, device=DEV) for _ in range(3)]
    p64.adjoint_force(*x, mass, cp, u, 0.7, b64)
    p32.adjoint_force_split(cell, off, mass, cp, [t.float() for t in u], 0.7, b32)
    assert rel(b32, b64) < 1e-4


def test_run_gradient_f32_matches_f64_and_finite_differences(pmpkg, O):
    """The differentiable-PM configuration on the FP32 path (128^3 on 128^3,
    32 KDK steps at dt = 0.01, checkpoint every 8): the FP32 gradient against
    the FP64 adjoint gradient of the same run (relative L2 < 1e-3) and
    against central differences of the FP64 loss on 64 random components
    (relative L2 < 1e-3)."""
    from pm_autograd import kdk_schedule, loss_fn, loss_fn_split

    ng = nrow = 128
    steps, dt, ckpt = 32, 0.01, 8
    psi0 = O.zeldovich_displacement(nrow, -2.0, seed=11)
    rms = np.sqrt(np.mean(np.sum(psi0 * psi0, axis=0)))
    psi_np = (psi0 * (0.5 / rms)).reshape(3, -1)
    q = lattice(ng, nrow)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    p64 = pmpkg.Plan(ng, "fp64", "spectral", 4)
    p32 = pmpkg.Plan(ng, "fp32", "spectral", 4)
    tpos, tvel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=12)
    tx, tv = [T(a) for a in tpos], [T(a) for a in tvel]
    for ck, dd in kdk_schedule(steps, dt)[:-1]:
        p64.step(*tx, *tv, mass, cp, ck, dd)
    target = p64.deposit(*tx, mass)[:, :, :ng].clone()

    psi64 = T(psi_np).requires_grad_(True)
    loss_fn(psi64, q, p64, ng, mass, cp, dt, steps, target, 1.0, ckpt).backward()
    psi32 = T(psi_np).requires_grad_(True)
    l32 = loss_fn_split(psi32, q, p32, ng, mass, cp, dt, steps, target, 1.0, ckpt)
    l32.backward()
    g64, g32 = psi64.grad.detach(), psi32.grad.detach()
    assert torch.isfinite(g32).all()
    e_adj = float((g32 - g64).norm() / g64.norm())
    assert e_adj < 1e-3, e_adj

    rng = np.random.default_rng(13)
    comps = [(int(rng.integers(3)), int(rng.integers(nrow ** 3))) for _ in range(64)]
    eps, fd, ad = 1e-5, [], []
    with torch.no_grad():
        for a, p in comps:
            base = psi64.detach().clone()
            base[a, p] += eps
            lp = float(loss_fn(base, q, p64, ng, mass, cp, dt, steps, target, 1.0, ckpt))
            base[a, p] -= 2 * eps
            lm = float(loss_fn(base, q, p64, ng, mass, cp, dt, steps, target, 1.0, ckpt))
            fd.append((lp - lm) / (2 * eps))
            ad.append(float(g32[a, p]))
    fd, ad = np.array(fd), np.array(ad)
    e_fd = np.linalg.norm(fd - ad) / np.linalg.norm(fd)
    assert e_fd < 1e-3, (e_fd, fd[:5], ad[:5])
