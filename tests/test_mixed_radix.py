"""Mesh sizes with factors 3 and 5 (2^a 3^b 5^c, the sizes the reference's
FFTE factorisation takes, src/fft/ffte1/factor.f:19-43): the generic radix
8/5/4/3/2 passes in both precisions against numpy.fft (pocketfft) and cuFFT,
the FP64 step against the CPU oracle, the FP32 split-position forces against
the FP64 oracle, and an FP64 adjoint dot-product test on a non-power-of-two
mesh.  Tolerances: FFT FP64 1e-13, FP32 2e-6 (relative L2); FP64 step 1e-12;
FP32 forces 1e-4 (the mixed-precision target); adjoint 1e-5 relative."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def rel(a, b):
    a, b = np.asarray(a), np.asarray(b)
    a = a.astype(np.complex128 if np.iscomplexobj(a) else np.float64)
    b = b.astype(np.complex128 if np.iscomplexobj(b) else np.float64)
    return float(np.linalg.norm((a - b).ravel()) / max(np.linalg.norm(b.ravel()), 1e-300))


def T(a, dtype=torch.float64):
    return torch.tensor(np.ascontiguousarray(a), dtype=dtype, device=DEV)


def H(t):
    return t.detach().cpu().numpy()


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("ng", [24, 40, 80, 120, 160, 240])
def test_fft_mixed_radix_vs_numpy(pmpkg, prec, ng):
    rng = np.random.default_rng(ng)
    x = rng.standard_normal((ng, ng, ng))
    plan = pmpkg.Plan(ng, prec)
    d = plan.new_mesh()
    d[:, :, :ng] = T(x, d.dtype)
    plan.fft_r2c(d)
    spec = H(d).view(np.complex128 if prec == "fp64" else np.complex64)
    ref = np.fft.rfftn(x.astype(np.float32).astype(np.float64) if prec == "fp32" else x)
    tol = 1e-13 if prec == "fp64" else 2e-6
    assert rel(spec, ref) < tol
    plan.fft_c2r(d)
    assert rel(H(d)[:, :, :ng] / ng ** 3, x) < tol
    assert np.all(H(d)[:, :, ng:] == 0)


@pytest.mark.parametrize("prec", ["fp64", "fp32"])
@pytest.mark.parametrize("ng", [384, 640, 960])
def test_fft_mixed_radix_large_vs_cufft(pmpkg, prec, ng):
    g = torch.Generator(device=DEV).manual_seed(ng)
    plan = pmpkg.Plan(ng, prec)
    d = plan.new_mesh()
    d[:, :, :ng] = torch.randn((ng, ng, ng), generator=g, device=DEV, dtype=d.dtype)
    x = d[:, :, :ng].double().clone()
    ref = torch.fft.rfftn(x)
    plan.fft_r2c(d)
    ours = torch.view_as_complex(d.view(ng, ng, ng // 2 + 1, 2)).to(torch.complex128)
    err = float((ours - ref).abs().norm() / ref.abs().norm())
    del ours, ref
    plan.fft_c2r(d)
    back = float((d[:, :, :ng].double() / ng ** 3 - x).norm() / x.norm())
    tol = 1e-13 if prec == "fp64" else 2e-6
    assert err < tol and back < tol, (err, back)
    del d, x
    torch.cuda.empty_cache()


@pytest.mark.parametrize("ng,nrow,kind,order", [(40, 40, "spectral", 4), (48, 32, "discrete", 2),
                                                (80, 40, "discrete", 4), (96, 48, "spectral", 2)])
def test_fp64_step_mixed_radix_vs_oracle(pmpkg, O, ng, nrow, kind, order):
    rng = np.random.default_rng(ng + nrow)
    x, y, z = (rng.uniform(0, ng, nrow ** 3) for _ in range(3))
    mass, cp, ck = ng ** 3 / nrow ** 3, 4 * np.pi, 0.01
    kid = 0 if kind == "discrete" else 1
    p = [np.zeros(nrow ** 3) for _ in range(3)]
    delta, phi, _ = O.force_step(ng, x, y, z, *p, mass, cp, ck, kid, order)
    plan = pmpkg.Plan(ng, "fp64", kind, order)
    tx = [T(a) for a in (x, y, z)]
    assert rel(H(plan.deposit(*tx, mass))[:, :, :ng], delta[:, :, :ng]) < 1e-13
    tp = [torch.zeros_like(tx[0]) for _ in range(3)]
    plan.step(*tx, *tp, mass, cp, ck, 0.0)
    plan.check()
    assert rel(H(plan.workspace_mesh())[:, :, :ng], phi[:, :, :ng]) < 1e-12
    assert rel(np.stack([H(a) for a in tp]), np.stack(p)) < 1e-12


@pytest.mark.parametrize("ng,nrow", [(40, 40), (80, 40), (160, 80)])
def test_fp32_forces_mixed_radix_within_1e4_of_fp64(pmpkg, O, ng, nrow):
    pos, vel = O.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=ng)
    mass, cp = ng ** 3 / nrow ** 3, 4 * np.pi
    f = [np.zeros(nrow ** 3) for _ in range(3)]
    O.force_step(ng, *(a.copy() for a in pos), *f, mass, cp, 1.0, 1, 4)
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*(T(a) for a in pos))
    v = [torch.zeros_like(off[0]) for _ in range(3)]
    plan.step_split(cell, off, v, mass, cp, 1.0, 0.0)  # v comes back as the force
    plan.check()
    err = rel(np.stack([H(a) for a in v]), np.stack(f))
    assert err < 1e-4, err


def test_fp64_adjoint_force_dot_product_mixed_radix(pmpkg):
    ng, np_ = 40, 6000
    rng = np.random.default_rng(7)
    x = [T(rng.uniform(2, ng - 2, np_)) for _ in range(3)]
    h = [T(rng.standard_normal(np_)) for _ in range(3)]
    u = [T(rng.standard_normal(np_)) for _ in range(3)]
    plan = pmpkg.Plan(ng, "fp64", "spectral", 4)
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


def test_unsupported_sizes_are_refused(pmpkg):
    for ng in (12, 36, 50, 100, 2048):
        with pytest.raises(pmpkg.PMError) as e:
            pmpkg.Plan(ng, "fp64")
        assert e.value.code == 2  # PM_ERR_SIZE
