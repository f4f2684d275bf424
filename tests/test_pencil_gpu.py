"""The pencil decomposition through its CUDA kernels, px x py pencils emulated
on one GPU (LocalExchange: the pencils run one after another and exchange by
device copies; no kernel waits on another pencil's).  Against the
undecomposed FP32 step (pm_step_f32) on the same particles:
  potential (the pencils' own rows assembled) within 1e-6 relative L2;
  velocities within 1e-5 relative L2 and positions within 1e-5 cells rms
  (1e-4 at most) after the steps (the FP32 sums of the two deposits differ
  in order);
  every particle on the pencil that owns its (x, y) cell, and some migrated.
And the first kick against the FP64 oracle's forces within 1e-4.
"""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def run_pair(pmpkg, ng, nrow, px, py, steps, dt, seed, peer=False):
    P = pmpkg.pencil
    cp, mass = 4 * np.pi, ng ** 3 / nrow ** 3
    pos, vel = pmpkg.zeldovich_ic(ng, nrow, -2.0, 0.5, seed=seed, device=DEV)
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*pos)
    v = [a.float() for a in vel]
    ids = torch.arange(nrow ** 3, dtype=torch.int32, device=DEV)
    pens = [P.Pencil(ng, px, py, r, "spectral", 4) for r in range(px * py)]
    parts = P.distribute(cell, off, v, ids, ng, px, py, range(px * py), cap_factor=2.0)
    n0 = [q.n for q in parts]
    ex = P.LocalPeerExchange(pens) if peer else P.LocalExchange()
    c1, o1, v1 = cell.clone(), [a.clone() for a in off], [a.clone() for a in v]
    for _ in range(steps):
        P.step(pens, parts, ex, mass, cp, dt, dt)
        plan.step_split(c1, o1, v1, mass, cp, dt, dt)
    for s in pens:
        s.check()
    plan.check()
    return plan, pens, parts, n0, (c1, o1, v1), (pos, vel)


def assemble(pens, ng):
    phi = torch.zeros((ng, ng, ng), dtype=torch.float64, device=DEV)
    for q in pens:
        phi[q.x0:q.x0 + q.nx, q.y0:q.y0 + q.ny] = q.potential()[:, :, :ng].double()
    return phi


@pytest.mark.parametrize("ng,nrow,px,py,peer", [(64, 64, 1, 1, False), (64, 64, 2, 2, False), (64, 64, 1, 4, False),
                                                (64, 64, 4, 2, False), (256, 128, 2, 4, False),
                                                (512, 128, 2, 2, False), (64, 64, 1, 1, True), (64, 64, 2, 2, True),
                                                (64, 64, 4, 2, True), (256, 128, 2, 4, True), (512, 128, 2, 2, True)])
def test_pencil_step_matches_single_box(pmpkg, ng, nrow, px, py, peer):
    """(peer: the transposes by the kernels' stores into the other pencils'
    buffers, LocalPeerExchange)"""
    P = pmpkg.pencil
    steps, dt = 3, (0.1 if ng <= 64 else 0.05)
    plan, pens, parts, n0, (c1, o1, v1), _ = run_pair(pmpkg, ng, nrow, px, py, steps, dt, seed=ng + px + 3 * py,
                                                      peer=peer)
    phi = assemble(pens, ng)
    phi1 = plan.workspace_mesh()[:, :, :ng].double()
    perr = float((phi - phi1).norm() / phi1.norm())
    assert perr < 1e-6, perr
    w = torch.cat([q.words[:, :q.n] for q in parts], dim=1)
    w = w[:, torch.argsort(w[7])]
    assert torch.equal(w[7], torch.arange(nrow ** 3, dtype=torch.int32, device=DEV))
    vel = torch.stack([w[4 + a].view(torch.float32) for a in range(3)]).double()
    vref = torch.stack(v1).double()
    verr = float((vel - vref).norm() / vref.norm())
    assert verr < 1e-5, verr
    xs = plan.join(w[0].contiguous(), [w[1 + a].view(torch.float32).contiguous() for a in range(3)])
    xr = plan.join(c1, o1)
    d = torch.stack([torch.remainder(a - b + ng / 2, ng) - ng / 2 for a, b in zip(xs, xr)])
    dmax, drms = float(d.abs().max()), float(d.pow(2).mean().sqrt())
    assert drms < 1e-5 and dmax < 1e-4, (drms, dmax)
    for s, q in zip(pens, parts):
        assert bool(torch.all(P.owner_of(q.cell[:q.n], ng, px, py) == s.rank))
    if px * py > 1 and ng <= 64:
        assert [q.n for q in parts] != n0, "no particle migrated"
    print(f"pencil ng={ng} nrow={nrow} {px}x{py}: potential {perr:.2e}, velocity {verr:.2e}, "
          f"position rms {drms:.2e} max {dmax:.2e}")
    for s in pens:
        s.close()
    plan.close()
    torch.cuda.empty_cache()


def test_pencil_first_kick_matches_oracle_forces(pmpkg, O):
    ng = nrow = 64
    dt = 0.25
    plan, pens, parts, _, _, (pos, vel) = run_pair(pmpkg, ng, nrow, 2, 2, 1, dt, seed=5)
    w = torch.cat([q.words[:, :q.n] for q in parts], dim=1)
    w = w[:, torch.argsort(w[7])]
    v = np.stack([w[4 + a].view(torch.float32).cpu().numpy() for a in range(3)]).astype(np.float64)
    v0 = np.stack([a.float().cpu().numpy() for a in vel]).astype(np.float64)
    f = [np.zeros(nrow ** 3) for _ in range(3)]
    O.force_step(ng, *(a.cpu().numpy().copy() for a in pos), *f, 1.0, 4 * np.pi, 1.0, 1, 4)
    err = np.linalg.norm((v - v0) / dt - np.stack(f)) / np.linalg.norm(np.stack(f))
    assert err < 1e-4, err


def test_pencil_rejects_bad_geometry(pmpkg):
    P = pmpkg.pencil
    for args in ((64, 3, 2, 0), (64, 32, 1, 0), (48, 2, 2, 0), (64, 2, 2, 4)):
        with pytest.raises(pmpkg.PMError):
            P.Pencil(*args)


def test_pencil_ranks_without_particles(pmpkg):
    """All particles in a clump inside pencil (0, 0) of 2 x 2: the other
    pencils deposit nothing, gather nothing and migrate nothing; the result
    still matches the undecomposed step."""
    P = pmpkg.pencil
    ng, px, py, n, dt = 64, 2, 2, 20000, 0.1
    g = torch.Generator(device="cpu").manual_seed(4)
    pos = [torch.rand(n, generator=g, dtype=torch.float64) * 6 + 5 for _ in range(2)]
    pos.append(torch.rand(n, generator=g, dtype=torch.float64) * ng)
    pos = [a.to(DEV) for a in pos]
    vel = [(torch.rand(n, generator=g) - 0.5).to(DEV) for _ in range(3)]
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    cell, off = plan.split(*pos)
    ids = torch.arange(n, dtype=torch.int32, device=DEV)
    pens = [P.Pencil(ng, px, py, r, "spectral", 4) for r in range(px * py)]
    parts = P.distribute(cell, off, vel, ids, ng, px, py, range(px * py), cap_factor=5.0)
    assert [q.n for q in parts] == [n, 0, 0, 0]
    c1, o1, v1 = cell.clone(), [a.clone() for a in off], [a.clone() for a in vel]
    mass, cp = ng ** 3 / n, 4 * np.pi
    for _ in range(2):
        P.step(pens, parts, P.LocalExchange(), mass, cp, dt, dt)
        plan.step_split(c1, o1, v1, mass, cp, dt, dt)
    for s in pens:
        s.check()
    phi = assemble(pens, ng)
    phi1 = plan.workspace_mesh()[:, :, :ng].double()
    assert float((phi - phi1).norm() / phi1.norm()) < 1e-6
    w = torch.cat([q.words[:, :q.n] for q in parts], dim=1)
    w = w[:, torch.argsort(w[7])]
    assert torch.equal(w[7], ids)
    vel_s = torch.stack([w[4 + a].view(torch.float32) for a in range(3)]).double()
    vref = torch.stack(v1).double()
    assert float((vel_s - vref).norm() / vref.norm()) < 1e-5
    for s in pens:
        s.close()
    plan.close()
