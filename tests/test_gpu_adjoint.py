"""Path-replay adjoint of the path tracer (lrt_render_adjoint) against finite differences.

* Linear functional F = sum_pixels <w, image> with fixed weights w: the adjoint (detached sampling)
  and the central difference of F at h = 1e-3 with common random numbers (the same samples at +h and
  -h) are estimates of the same dE[F]/dparam. Over independent sample ranges (seeds):
  - every parameter: the two means agree within 3 Monte Carlo standard errors (of the two estimates,
    from their spread over the seeds), with no other allowance;
  - parameters that no sampling decision depends on (diffuse albedos, conductor eta / k, the coat tints)
    also agree path by path: their paired difference is float32 rounding of the images and the
    adjoint's sums, so its mean is within 3 of its own (much smaller) standard errors plus 2e-5 of the
    gradient (measured: at most 1.1e-5).
  Where a sampling decision depends on the parameter (GGX directions on alpha, the plastic lobe choice
  on the albedo's luminance), the difference quotient moves by rare, large jumps where a decision flips
  between +h and -h: its mean is right but its spread needs many seeds. 16 seeds for the path-by-path
  set, 96 for all 38 parameters of the differentiation workload. Both run without Russian roulette,
  whose survival probability follows the throughput and would add such jumps to every parameter.
* The same against central differences of the reference CPU renderer (oracle/_ref) on the rough
  conductor, rough plastic and rough coating scenes, their roughness among the parameters.
* Materials moved by lrt_scene_update_materials render exactly as a fresh upload of the moved scene.
* An L2 image loss optimised with Adam through the autograd wrapper decreases and moves the
  roughness toward the target.
"""
import numpy as np
import pytest
import torch

import diff
import oracle
import scenes
from diff_harness import render

pytestmark = pytest.mark.gpu

DEPTH, RR = 6, 3
NO_RR = DEPTH  # roulette from depth >= max_depth: never


def fd_jobs(scene, sphere, index, w, h, spp, seeds):
    """one job per (seed, material) with the sphere carrying each material, packed back to back"""
    jobs, off = [], 0
    for k in range(seeds):
        for name in scenes.MATERIAL_NAMES:
            jobs.append(scenes.job_desc(scene.camera, w, h, spp, k * spp, sphere, index[name], off))
            off += 3 * w * h
    return jobs, off


PATH_BY_PATH_REL = 2e-5


def assert_agree(adj, fd, names, sharp=()):
    """adj, fd: [seeds, params] estimates on the same samples. Every parameter's means within 3 Monte Carlo
    standard errors; the columns in `sharp` also path by path (paired mean difference within 3 of its
    standard errors + PATH_BY_PATH_REL of the gradient)."""
    n = adj.shape[0]
    diff_mean = adj.mean(axis=0) - fd.mean(axis=0)
    se_mc = np.sqrt(adj.var(axis=0, ddof=1) / n + fd.var(axis=0, ddof=1) / n)
    d = adj - fd
    se_d = d.std(axis=0, ddof=1) / np.sqrt(n)
    msgs = []
    for j in range(adj.shape[1]):
        if abs(diff_mean[j]) > 3.0 * se_mc[j]:
            msgs.append("%s: adj %.6g fd %.6g, %.2f Monte Carlo SE" % (
                names[j], adj[:, j].mean(), fd[:, j].mean(), abs(diff_mean[j]) / max(se_mc[j], 1e-300)))
        if j in sharp and abs(diff_mean[j]) > 3.0 * se_d[j] + PATH_BY_PATH_REL * abs(fd[:, j].mean()):
            msgs.append("%s: path by path adj %.8g fd %.8g (relative %.2e, paired SE %.2e)" % (
                names[j], adj[:, j].mean(), fd[:, j].mean(), diff_mean[j] / abs(fd[:, j].mean()), se_d[j]))
    assert not msgs, "\n".join(msgs)


def central_differences(ctx, dm, jobs, floats, seeds, weights, step, params):
    """per seed, (F(+h) - F(-h)) / 2h for the parameter indices `params` (all seeds in one batch)"""
    per = floats // seeds
    base = dm.values()
    fd = np.zeros((seeds, len(params)))
    for col, j in enumerate(params):
        f = []
        for sign in (1.0, -1.0):
            v = base.copy()
            v[j] += sign * step
            dm.set_values(v, setup=False)
            img = ctx.render_batch(jobs, DEPTH, NO_RR)
            f.append((img[:floats] * weights).astype(np.float64).reshape(seeds, per).sum(axis=1))
        fd[:, col] = (f[0] - f[1]) / (2 * step)
    dm.set_values(base)
    return fd


def adjoint_per_seed(dm, jobs, seeds, weights):
    return np.stack([dm.adjoint(jobs[k * 7:(k + 1) * 7], DEPTH, NO_RR, weights) for k in range(seeds)])


@pytest.fixture(scope="module")
def library3():
    return scenes.open_box_library(level=3)


def sharp_params(scene, params):
    """parameters no sampling decision depends on: diffuse albedos, conductor eta / k, coat tints"""
    return [j for j, (m, field, c) in enumerate(params)
            if field in ("eta", "k", "specular_reflectance") or scene.materials[m]["type"] == diff.abi.MAT_DIFFUSE]


def test_adjoint_matches_central_differences_path_by_path(ctx, library3):
    scene, sphere, index = library3
    ctx.upload(scene)
    dm = diff.Differentiable(ctx, scene)
    assert len(dm.params) == 38
    sharp = sharp_params(scene, dm.params)
    assert len(sharp) == 24
    seeds = 16
    jobs, floats = fd_jobs(scene, sphere, index, 20, 20, 4, seeds)
    weights = np.random.default_rng(7).uniform(0.5, 1.5, floats).astype(np.float32)
    adj = adjoint_per_seed(dm, jobs, seeds, weights)[:, sharp]
    fd = central_differences(ctx, dm, jobs, floats, seeds, weights, 1e-3, sharp)
    assert np.abs(adj).min() > 0
    assert_agree(adj, fd, [dm.names()[j] for j in sharp], sharp=range(len(sharp)))


def test_adjoint_matches_central_differences_all(ctx, library3):
    scene, sphere, index = library3
    ctx.upload(scene)
    dm = diff.Differentiable(ctx, scene)
    seeds = 96
    jobs, floats = fd_jobs(scene, sphere, index, 20, 20, 4, seeds)
    weights = np.random.default_rng(7).uniform(0.5, 1.5, floats).astype(np.float32)
    adj = adjoint_per_seed(dm, jobs, seeds, weights)
    fd = central_differences(ctx, dm, jobs, floats, seeds, weights, 1e-3, list(range(len(dm.params))))
    assert np.all(np.abs(adj).max(axis=0) > 0), "a parameter without any derivative"
    assert_agree(adj, fd, dm.names(), sharp=sharp_params(scene, dm.params))


def test_adjoint_zero_and_linear(ctx):
    scene, sphere, index = scenes.open_box_library(level=3)
    ctx.upload(scene)
    dm = diff.Differentiable(ctx, scene)
    jobs, floats = fd_jobs(scene, sphere, index, 16, 16, 4, 1)
    assert np.all(dm.adjoint(jobs, DEPTH, RR, np.zeros(floats, np.float32)) == 0.0)
    w = np.random.default_rng(3).uniform(-1, 1, floats).astype(np.float32)
    g1 = dm.adjoint(jobs, DEPTH, RR, w)
    g2 = dm.adjoint(jobs, DEPTH, RR, 2 * w)
    np.testing.assert_allclose(g2, 2 * g1, rtol=1e-4, atol=1e-9 * np.abs(g1).max())


def test_update_materials_equals_fresh_upload(ctx):
    scene, sphere, index = scenes.open_box_library(level=3)
    ctx.upload(scene)
    dm = diff.Differentiable(ctx, scene)
    v = dm.values()
    v = v * np.random.default_rng(11).uniform(0.8, 1.1, v.size)
    dm.set_values(v)
    jobs, _ = fd_jobs(scene, sphere, index, 16, 12, 3, 1)
    moved = ctx.render_batch(jobs, DEPTH, RR)
    scene.materials = diff.with_values(scene.materials, dm.params, v)
    ctx.upload(scene)
    fresh = ctx.render_batch(jobs, DEPTH, RR)
    assert np.array_equal(moved, fresh)


@pytest.mark.skipif(not oracle.reference_available(), reason="reference build (oracle/_ref) missing")
@pytest.mark.parametrize("material", ["rough_conductor", "rough_plastic", "rough_coating"])
def test_adjoint_matches_reference_differences(ctx, material):
    """central differences of the reference CPU renderer (same samples at +h and -h, h = 1e-3) on the open
    box with the sphere in `material`: the sphere's roughness (for the rough coating also its nested
    rough glass), its other parameters, and the white wall's albedo[0]; within 3 Monte Carlo standard
    errors (the GPU and CPU renders are not bit-identical, so no path-by-path bar)"""
    scene = scenes.open_box(material, level=3)
    ctx.upload(scene)
    sphere_params = [p for p in diff.scene_params(scene.materials) if p[0] >= 3]
    params = sphere_params + [(0, "diffuse_reflectance", 0)]
    if material == "rough_conductor":
        params = [p for p in params if p[1] in ("alpha", "diffuse_reflectance") or p[2] in (0, 2)]
    dm = diff.Differentiable(ctx, scene, params)
    seeds, w, h, spp = 32, 12, 12, 4
    weights = np.random.default_rng(5).uniform(0.5, 1.5, (h, w, 3)).astype(np.float32)
    base = dm.values()
    adj = np.zeros((seeds, len(params)))
    fd = {1e-3: np.zeros((seeds, len(params)))}
    worlds = {}
    for j in range(len(params)):
        for step in fd:
            for sign in (1.0, -1.0):
                v = base.copy()
                v[j] += sign * step
                moved = scenes.Scene(scene.objects, diff.with_values(scene.materials, params, v), scene.emitters,
                                     scene.camera, scene.name)
                worlds[(j, step, sign)] = oracle.RefWorld(moved)
    for k in range(seeds):
        job = scenes.job_desc(scene.camera, w, h, spp, k * spp)
        adj[k] = dm.adjoint([job], DEPTH, NO_RR, weights)
        p = scenes.render_params(w, h, spp, DEPTH, NO_RR, sample_offset=k * spp)
        for j in range(len(params)):
            for step, arr in fd.items():
                fp = float((worlds[(j, step, 1.0)].render(p)[0] * weights).astype(np.float64).sum())
                fm = float((worlds[(j, step, -1.0)].render(p)[0] * weights).astype(np.float64).sum())
                arr[k, j] = (fp - fm) / (2 * step)
    for wld in worlds.values():
        wld.close()
    assert any(p[1] == "alpha" for p in params)
    assert_agree(adj, fd[1e-3], dm.names())


def test_adam_moves_roughness_to_target(ctx):
    """target at alpha 0.3; start at alpha 0.6 for every rough material; Adam (lr 0.01) on the alphas
    with an L2 image loss. The noisy per-step loss is not a progress measure (smoother surfaces give
    spikier sun highlights, so more noise at the target); the parameters and a high-spp loss are."""
    scene, sphere, index = scenes.open_box_library(level=3)
    ctx.upload(scene)
    alphas = [p for p in diff.scene_params(scene.materials) if p[1] == "alpha"]
    dm = diff.Differentiable(ctx, scene, alphas)
    w, h, spp = 24, 24, 8
    jobs, floats = fd_jobs(scene, sphere, index, w, h, spp, 1)

    def moved(base_jobs, spp_, offset):
        return [scenes.job_desc(scene.camera, w, h, spp_, offset, j.override_object, j.override_material,
                                j.output_offset) for j in base_jobs]

    dm.set_values(np.full(len(alphas), 0.3), setup=False)
    target = torch.from_numpy(ctx.render_batch(moved(jobs, 256, 1 << 20), DEPTH, RR).astype(np.float64))

    def clean_loss(vals):
        dm.set_values(vals, setup=False)
        img = torch.from_numpy(ctx.render_batch(moved(jobs, 128, 1 << 22), DEPTH, RR).astype(np.float64))
        return float(((img - target) ** 2).mean())

    start = np.full(len(alphas), 0.6)
    loss_start = clean_loss(start)
    values = torch.tensor(start, dtype=torch.float64, requires_grad=True)
    opt = torch.optim.Adam([values], lr=0.01)
    for it in range(60):
        opt.zero_grad()
        img = render(values, dm, moved(jobs, spp, 1000 * it), moved(jobs, spp, 1000 * it + 500), DEPTH, RR)
        loss = ((img - target) ** 2).mean()
        loss.backward()
        opt.step()
        with torch.no_grad():
            values.clamp_(0.05, 1.0)
    final = values.detach().numpy()
    loss_end = clean_loss(final)
    assert np.abs(final - 0.3).mean() < 0.5 * np.abs(start - 0.3).mean(), final
    assert loss_end < loss_start, (loss_start, loss_end)


@pytest.mark.parametrize("cap", [1 << 21, 4096])
def test_wavefront_adjoint_equals_megakernel(ctx, library3, cap):
    """the wavefront adjoint (per-depth records, suffix pass per wave) and the one-thread-per-path
    kernel replay the same paths; with roulette on and, at the small capacity, pixels split across
    waves, their gradients differ only by float summation order"""
    scene, sphere, index = library3
    ctx.upload(scene)
    dm = diff.Differentiable(ctx, scene)
    jobs, floats = fd_jobs(scene, sphere, index, 24, 20, 6, 1)
    w = np.random.default_rng(9).uniform(-1, 1, floats).astype(np.float32)
    try:
        ctx.set_option("wave_capacity", cap)
        wave = dm.adjoint(jobs, DEPTH, RR, w)
        ctx.set_option("adjoint_megakernel", 1)
        mega = dm.adjoint(jobs, DEPTH, RR, w)
    finally:
        ctx.set_option("adjoint_megakernel", 0)
        ctx.set_option("wave_capacity", 1 << 21)
    assert np.abs(mega).max() > 0
    np.testing.assert_allclose(wave, mega, rtol=1e-3, atol=1e-5 * np.abs(mega).max())
