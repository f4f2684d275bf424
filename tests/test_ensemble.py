"""Batched ensemble of boxes with mixed mesh sizes (32 to 128): one CUDA
graph of a KDK run versus each box advanced alone with its own FP32 plan
through the same schedule; the eager step versus the graph; the autotuner's
cache file."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

DEV = "cuda:0"


@pytest.fixture(scope="module", autouse=True)
def _cuda():
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")


def boxes_state(pmpkg, sizes, seeds):
    cells, offs, vels = [], [[], [], []], [[], [], []]
    for ng, sd in zip(sizes, seeds):
        pos, vel = pmpkg.zeldovich_ic(ng, ng, -1.5 - 0.1 * (sd % 5), 0.3 + 0.1 * (sd % 7), seed=sd, device=DEV)
        plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
        c, o = plan.split(*pos)
        cells.append(c)
        for a in range(3):
            offs[a].append(o[a])
            vels[a].append(vel[a].float())
    return torch.cat(cells), [torch.cat(x) for x in offs], [torch.cat(x) for x in vels]


def solo(pmpkg, sizes, cell, off, vel, cp, dt, steps):
    """Each box alone through the same merged-KDK schedule."""
    out_c, out_o, out_v = cell.clone(), [t.clone() for t in off], [t.clone() for t in vel]
    start = 0
    for ng in sizes:
        n = ng ** 3
        plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
        sl = slice(start, start + n)
        c = out_c[sl].clone()
        o = [t[sl].clone() for t in out_o]
        v = [t[sl].clone() for t in out_v]
        for s in range(steps + 1):
            ck = 0.5 * dt if s in (0, steps) else dt
            plan.step_split(c, o, v, 1.0, cp, ck, dt if s < steps else 0.0)
        out_c[sl] = c
        for a in range(3):
            out_o[a][sl] = o[a]
            out_v[a][sl] = v[a]
        start += n
    return out_c, out_o, out_v


def test_ensemble_graph_matches_boxes_alone(pmpkg, tmp_path):
    sizes = [32, 48, 64, 32, 96, 48, 128]
    seeds = [5, 6, 7, 8, 9, 10, 11]
    cp, dt, steps = 4 * np.pi, 0.01, 3
    cell, off, vel = boxes_state(pmpkg, sizes, seeds)
    ref_c, ref_o, ref_v = solo(pmpkg, sizes, cell, off, vel, cp, dt, steps)
    cache = tmp_path / "tune.txt"
    ens = pmpkg.Ensemble(sizes, [n ** 3 for n in sizes], [1.0] * len(sizes), tune_cache=str(cache))
    info = ens.info()
    assert sorted(c["ng"] for c in info["classes"]) == [32, 48, 64, 96, 128]
    assert cache.exists() and len(cache.read_text().splitlines()) == 5
    c, o, v = cell.clone(), [t.clone() for t in off], [t.clone() for t in vel]
    ens.run(c, o, v, cp, dt, steps)
    torch.cuda.synchronize()
    assert ens.info()["graph_nodes"] > 0
    dv = max(float((a - b).abs().max()) for a, b in zip(v, ref_v))
    assert dv < 1e-4 * max(float(t.abs().max()) for t in ref_v)
    moved = (c != ref_c).float().mean()
    assert float(moved) < 1e-3  # cells agree except for particles within rounding of a face
    # eager steps give the same state as the graph
    c2, o2, v2 = cell.clone(), [t.clone() for t in off], [t.clone() for t in vel]
    for s in range(steps + 1):
        ck = 0.5 * dt if s in (0, steps) else dt
        ens.step(c2, o2, v2, cp, ck, dt if s < steps else 0.0)
    torch.cuda.synchronize()
    assert max(float((a - b).abs().max()) for a, b in zip(v2, v)) < 1e-4 * max(float(t.abs().max()) for t in v)
    # a second ensemble reads its tile widths and radix splits from the cache
    ens2 = pmpkg.Ensemble(sizes, [n ** 3 for n in sizes], [1.0] * len(sizes), tune_cache=str(cache))
    shape = lambda i: [(c["tile_cols"], c["radix1"]) for c in i["classes"]]  # noqa: E731
    assert shape(ens2.info()) == shape(info)
    # a hand-written cache line (the old five-field form too) is taken as given
    gpu = cache.read_text().split()[0]
    cache.write_text(f"{gpu} 32 1 4 16 1\n{gpu} 64 1 4 8\n")
    ens3 = pmpkg.Ensemble([32, 64], [32 ** 3, 64 ** 3], [1.0, 1.0], tune_cache=str(cache))
    got = {c["ng"]: (c["tile_cols"], c["radix1"]) for c in ens3.info()["classes"]}
    assert got == {32: (16, 2), 64: (8, 8)}


@pytest.mark.parametrize("ng", [16, 32, 64, 128])
def test_fft_shapes_agree(pmpkg, ng):
    """Every tile width x radix split the autotuner may pick gives the same
    Poisson solution as the default shape (FP32 rounding)."""
    g = torch.Generator(device="cuda").manual_seed(ng)
    x = torch.randn((ng, ng, ng), generator=g, device="cuda")
    plan = pmpkg.Plan(ng, "fp32", "spectral", 4)
    ref = plan.new_mesh()
    ref[:, :, :ng] = x
    plan.poisson(ref, 2.0)
    default_r1 = {16: 4, 32: 4, 64: 8, 128: 8}[ng]
    alt_r1 = {16: 2, 32: 2, 64: 4, 128: 4}[ng]
    for tk in (0, 8, 16, 32):
        for r1 in (default_r1, alt_r1):
            plan.set_fft_shape(tk, r1)
            m = plan.new_mesh()
            m[:, :, :ng] = x
            plan.poisson(m, 2.0)
            err = float((m[:, :, :ng] - ref[:, :, :ng]).norm() / ref[:, :, :ng].norm())
            assert err < 1e-6, (tk, r1, err)
    with pytest.raises(pmpkg.PMError):
        plan.set_fft_shape(12, 0)
    with pytest.raises(pmpkg.PMError):
        plan.set_fft_shape(0, 3)


def test_dealt_boxes_match_the_whole_ensemble(pmpkg):
    """Boxes dealt to two ranks (slab.deal_boxes, as bench.py --gpus 2 does):
    each rank's ensemble of its own boxes gives those boxes the state the
    whole ensemble gives them (independent boxes; FP32 rounding)."""
    sizes = [32, 64, 48, 128, 32, 96, 64, 48]
    seeds = list(range(20, 28))
    cp, dt, steps = 4 * np.pi, 0.01, 2
    cell, off, vel = boxes_state(pmpkg, sizes, seeds)
    whole = pmpkg.Ensemble(sizes, [n ** 3 for n in sizes], [1.0] * len(sizes), autotune=False)
    wc, wo, wv = cell.clone(), [t.clone() for t in off], [t.clone() for t in vel]
    whole.run(wc, wo, wv, cp, dt, steps)
    starts = np.cumsum([0] + [n ** 3 for n in sizes])
    deal = pmpkg.slab.deal_boxes([n ** 3 for n in sizes], 2)
    assert sorted(b for d in deal for b in d) == list(range(len(sizes)))
    for mine in deal:
        idx = torch.cat([torch.arange(int(starts[b]), int(starts[b + 1]), device=DEV) for b in mine])
        c, o, v = cell[idx].clone(), [t[idx].clone() for t in off], [t[idx].clone() for t in vel]
        ens = pmpkg.Ensemble([sizes[b] for b in mine], [sizes[b] ** 3 for b in mine], [1.0] * len(mine),
                             autotune=False)
        ens.run(c, o, v, cp, dt, steps)
        torch.cuda.synchronize()
        dv = max(float((a - b[idx]).abs().max()) for a, b in zip(v, wv))
        assert dv < 1e-4 * max(float(t.abs().max()) for t in wv), dv
        assert float((c != wc[idx]).float().mean()) < 1e-3


@pytest.mark.parametrize("ng", [32, 64, 128])
def test_every_shape_gives_the_same_run(pmpkg, tmp_path, ng):
    """A 10-step KDK run of an ensemble under every strided-pass shape the
    autotuner may pick (forced through the cache file) ends in the state the
    default shape gives: velocities within 1e-4 of their scale, cells equal
    but for rounding at a face."""
    sizes = [ng, ng, ng]
    cell, off, vel = boxes_state(pmpkg, sizes, [31, 32, 33])
    cp, dt, steps = 4 * np.pi, 0.01, 10
    gpu = None
    ref = None
    default_r1 = {32: 4, 64: 8, 128: 8}[ng]
    for tk in (0, 8, 16, 32):
        for rv, r1 in ((0, default_r1), (1, {32: 2, 64: 4, 128: 4}[ng])):
            cache = tmp_path / f"c{tk}_{rv}.txt"
            if gpu is None:
                probe = pmpkg.Ensemble([ng], [ng ** 3], [1.0], autotune=True, tune_cache=str(tmp_path / "probe.txt"))
                gpu = (tmp_path / "probe.txt").read_text().split()[0]
                probe.close()
            cache.write_text(f"{gpu} {ng} 1 4 {tk} {rv}\n")
            ens = pmpkg.Ensemble(sizes, [n ** 3 for n in sizes], [1.0] * 3, autotune=False, tune_cache=str(cache))
            got = {c["ng"]: (c["tile_cols"], c["radix1"]) for c in ens.info()["classes"]}
            assert got == {ng: (tk, r1)}
            c, o, v = cell.clone(), [t.clone() for t in off], [t.clone() for t in vel]
            ens.run(c, o, v, cp, dt, steps)
            torch.cuda.synchronize()
            ens.close()
            if ref is None:
                ref = (c, v)
                continue
            scale = max(float(t.abs().max()) for t in ref[1])
            dv = max(float((a - b).abs().max()) for a, b in zip(v, ref[1]))
            assert dv < 1e-4 * scale, (tk, r1, dv / scale)
            assert float((c != ref[0]).float().mean()) < 1e-3, (tk, r1)
