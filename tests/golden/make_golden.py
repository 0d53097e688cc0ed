"""Generates the golden fixtures in tests/golden/ from the reference itself.

Run in a tree where the reference is available (oracle/_ref/libpxref_ieee.so
built by `make -C oracle`):

    python tests/golden/make_golden.py

Every output comes from the reference's own public functions (projectSplats,
rasterizeSplats, photometricLoss, meanSsim, rasterizeSplatsBackward,
densifyAndPrune, SplatTrainer), compiled from its sources with IEEE
arithmetic. The per-tile key lists are derived from the reference's projected
splats with buildTiles' rule (SplatRaster.cpp:114-151), which the
oracle pin test shows composites to the reference's image bit for bit.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.dirname(HERE))
sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))

import oracle_lib as O  # noqa: E402
from parallax_b200._abi import RasterOptions, TrainConfig  # noqa: E402


def view_arrays(view):
    return dict(K=np.array(view.K, dtype=np.float64), size=np.array([view.width, view.height]),
                R=np.asarray(view.R, dtype=np.float64), t=np.asarray(view.t, dtype=np.float64))


def options_arrays(opt: RasterOptions):
    return dict(background=np.array(list(opt.background), dtype=np.float32),
                sh_degree=np.int32(opt.sh_degree), min_alpha=np.float32(opt.min_alpha),
                transmittance_cutoff=np.float32(opt.transmittance_cutoff),
                screen_dilation=np.float32(opt.screen_dilation))


def projected_arrays(p):
    return {f"proj_{name}": p[name] for name in p.dtype.names}


def raster_case(name, sh_degree, count, width, height, seed, background=(0.0, 0.0, 0.0)):
    params, rest = O.random_cloud(seed, count, sh_degree, log_scale_mean=-3.2)
    view = O.orbit_views(2, width, height, seed=seed)[1]
    opt = RasterOptions(sh_degree=sh_degree, background=background)
    proj = O.ref_project(params, rest, sh_degree, view, opt)
    proj = np.sort(proj, order=["depth", "index"])
    offsets, entries = O.oracle_tiles(proj, width, height)
    gaussian_entries = proj["index"][entries].astype(np.int32)
    rgb, T = O.ref_render(params, rest, sh_degree, view, opt)
    rgb_from_list, _ = O.ref_rasterize(proj, view, opt)
    assert np.array_equal(rgb, rgb_from_list)
    target = np.random.default_rng(seed + 100).uniform(0, 1, rgb.shape).astype(np.float32)
    loss, dL = O.ref_loss(rgb, target, width, height, 0.2)
    ssim, dssim = O.ref_ssim(rgb, target, width, height)
    grads, screen, visible = O.ref_backward(params, rest, sh_degree, view, opt, dL)
    np.savez_compressed(
        os.path.join(HERE, f"{name}.npz"), params=params, rest=np.int32(rest),
        cloud_sh_degree=np.int32(sh_degree), **view_arrays(view), **options_arrays(opt),
        **projected_arrays(proj), tile_offsets=offsets, tile_entries=gaussian_entries,
        rgb=rgb, transmittance=T, target=target, ssim_weight=np.float32(0.2),
        loss=np.float32(loss), dL_drgb=dL, ssim=np.float32(ssim), d_ssim=dssim, grads=grads,
        screen_gradient=screen, visible_count=visible)
    print(name, "visible", len(proj), "pairs", len(entries), "loss", loss)


def ties_case():
    """A cloud whose gaussians sit on 30 depth planes (camera along +z, so
    every gaussian of a plane projects to a bit-equal depth), many of them
    overlapping on screen. The reference orders equal depths with the unstable
    std::sort (SplatRaster.cpp:260-261), so this fixture records its own
    order as it comes out of projectSplats (`proj_*` unsorted), the tile lists
    buildTiles' rule (SplatRaster.cpp:114-151) derives from that order, its
    image, and, for the specified order (equal depths by gaussian index), the
    reference's arithmetic on its own projections re-sorted that way: image,
    loss and gradients."""
    sh, count, width, height = 3, 900, 96, 72
    params, rest = O.random_cloud(77, count, sh, log_scale_mean=-3.0)
    rs = np.random.default_rng(5)
    levels = rs.uniform(-0.6, 0.6, 30).astype(np.float32)
    params[2] = levels[rs.integers(0, 30, count)]
    params[0] = rs.uniform(-0.5, 0.5, count)
    params[1] = rs.uniform(-0.4, 0.4, count)
    # a few exact duplicates: fully coincident tied splats
    params[:, 850:] = params[:, 800:850]
    view = O.make_view(width, height, 2.5)
    opt = RasterOptions(sh_degree=sh, background=(0.1, 0.2, 0.3))
    proj = O.ref_project(params, rest, sh, view, opt)
    offsets, entries = O.oracle_tiles(proj, width, height)
    rgb, T = O.ref_render(params, rest, sh, view, opt)
    rgb_from_list, _ = O.ref_rasterize(proj, view, opt)
    assert np.array_equal(rgb, rgb_from_list)
    target = np.random.default_rng(78).uniform(0, 1, rgb.shape).astype(np.float32)
    ordered = O.tie_ordered(proj)
    loss_i, rgb_i, grads_i, screen_i, visible_i = O.ref_render_and_accumulate_projected(
        params, rest, sh, view, opt, ordered, target, 0.2)
    d = proj["depth"].view(np.uint32)
    runs = [(b, e) for b, e in O.tie_runs(d) if e - b > 1]
    scrambled = sum(not np.all(np.diff(proj["index"][b:e]) > 0) for b, e in runs)
    assert scrambled > 0, "the reference kept index order in every tie run"
    np.savez_compressed(
        os.path.join(HERE, "ties.npz"), params=params, rest=np.int32(rest),
        cloud_sh_degree=np.int32(sh), **view_arrays(view), **options_arrays(opt),
        **projected_arrays(proj), tile_offsets=offsets,
        tile_entries=proj["index"][entries].astype(np.int32), rgb=rgb, transmittance=T,
        target=target, ssim_weight=np.float32(0.2), index_order_rgb=rgb_i,
        index_order_loss=np.float32(loss_i), index_order_grads=grads_i,
        index_order_screen_gradient=screen_i, index_order_visible_count=visible_i)
    print("ties: visible", len(proj), "tie runs", len(runs), "scrambled by std::sort", scrambled,
          "pairs", len(entries))


def c1_run_case():
    """The plain CPU-runnable configuration end to end under the reference's own
    trainer (SplatTrainer.cpp:326-362): 20k gaussians SH0 (start cloud seed 2),
    16 cameras on a radius-3 sphere at 320x240 (seed 3), targets rendered by
    the reference from the truth cloud (seed 1) and quantised to 8-bit frames
    (stored, and trained on as frame / 255), 200 iterations of one view, the
    reference's default schedule otherwise. Records the loss of every
    iteration and the final cloud's PSNR over the 16 views."""
    import parallax_b200 as px
    from parallax_b200.scenes import workload_scene

    truth, start, views = workload_scene("c1")
    opt = RasterOptions(sh_degree=0)
    oviews = [O.View(tuple(v.K), v.width, v.height, np.asarray(v.R), np.asarray(v.t))
              for v in views]
    frames = []
    for v in oviews:
        rgb, _ = O.ref_render(truth.params, 0, 0, v, opt)
        frames.append(np.rint(np.clip(rgb, 0, 1) * 255.0).astype(np.uint8))
    images = [f.astype(np.float32) / np.float32(255.0) for f in frames]
    cfg = TrainConfig(iterations=200, sh_degree=0)
    trainer = O.RefTrainer(start.params, 0, 0, oviews, images, cfg)
    losses = []
    while trainer.step():
        losses.append(trainer.state()["last_loss"])
    final = trainer.cloud()
    psnr = []
    for v, im in zip(oviews, images):
        rgb, _ = O.ref_render(final, 0, 0, v, opt)
        mse = float(np.mean((np.clip(rgb, 0, 1).astype(np.float64) - im) ** 2))
        psnr.append(10.0 * np.log10(1.0 / mse))
    arrays = {}
    for i, v in enumerate(oviews):
        for k, a in view_arrays(v).items():
            arrays[f"view{i}_{k}"] = a
    # the start cloud is not stored: pxs_synthetic_cloud(2, 20000, 0) regenerates
    # it (tests/test_ref_bench.py pins that generator to the reference's Rng)
    np.savez_compressed(os.path.join(HERE, "c1_run.npz"), frames=np.stack(frames),
                        losses=np.array(losses, np.float32), psnr=np.array(psnr),
                        n_views=np.int32(len(oviews)), **arrays)
    print("c1 run: final loss", losses[-1], "mean PSNR", float(np.mean(psnr)), "count",
          final.shape[1])
    assert px is not None


def densify_case():
    params, rest = O.random_cloud(21, 600, 1, log_scale_mean=-3.0)
    rs = np.random.default_rng(22)
    screen = rs.uniform(0, 1e-3, params.shape[1]).astype(np.float32)
    visible = rs.integers(0, 3, params.shape[1]).astype(np.int32)
    cases = {}
    for tag, iteration, max_g in [("a", 600, 600000), ("b", 4000, 600000), ("c", 600, 800)]:
        cfg = TrainConfig(max_gaussians=max_g)
        out, source, state, counts = O.ref_densify(params, rest, screen, visible, cfg, 3.3,
                                                   iteration, 7)
        cases.update({f"{tag}_iteration": np.int32(iteration), f"{tag}_max": np.int32(max_g),
                      f"{tag}_params": out, f"{tag}_source": source,
                      f"{tag}_rng": np.uint32(state), f"{tag}_counts": np.array(counts)})
        print("densify", tag, out.shape, counts)
    np.savez_compressed(os.path.join(HERE, "densify.npz"), params=params, rest=np.int32(rest),
                        screen_gradient=screen, visible_count=visible,
                        extent=np.float32(3.3), rng=np.uint32(7), **cases)


def trainer_case():
    """The reference trainer's blob scene (SplatTrainerTest.cpp:15-99) for 60
    iterations with densification every 20, one view per step."""
    truth, _ = O.truth_cloud()
    views = O.ring_of_views(4, 1.6, 24, 24)
    images = [O.ref_render(truth, 0, 0, v, RasterOptions())[0] for v in views]
    start, rest = O.rough_start(12)
    cfg = TrainConfig(iterations=60, sh_degree=0, sh_increase_interval=0,
                      densify_from_iteration=20, densify_until_iteration=60, densify_interval=20,
                      densify_grad_threshold=0.0, opacity_reset_interval=0)
    trainer = O.RefTrainer(start, rest, 0, views, images, cfg)
    losses, counts = [], []
    while trainer.step():
        st = trainer.state()
        losses.append(st["last_loss"])
        counts.append(st["count"])
    final = trainer.cloud()
    st = trainer.state()
    finished, sh = trainer.finish()
    arrays = {}
    for i, v in enumerate(views):
        for k, a in view_arrays(v).items():
            arrays[f"view{i}_{k}"] = a
        arrays[f"image{i}"] = images[i]
    cfg_fields = {f"cfg_{name}": np.array(getattr(cfg, name)) for name, _ in cfg._fields_}
    np.savez_compressed(os.path.join(HERE, "trainer_blobs.npz"), start=start,
                        n_views=np.int32(len(views)), losses=np.array(losses, np.float32),
                        counts=np.array(counts, np.int32), final=final, finished=finished,
                        smoothed=np.float32(st["smoothed_loss"]), extent=np.float32(st["extent"]),
                        **arrays, **cfg_fields)
    print("trainer", final.shape, finished.shape, losses[0], losses[-1])


def main():
    O.build_oracle()
    if sys.argv[1:] == ["ties"]:
        ties_case()
        return
    if sys.argv[1:] == ["c1"]:
        c1_run_case()
        return
    assert O.ref_available("ieee"), "oracle/_ref/libpxref_ieee.so is required"
    raster_case("raster_sh0", 0, 700, 64, 48, seed=31)
    raster_case("raster_sh3", 3, 500, 48, 40, seed=32, background=(0.2, 0.3, 0.4))
    ties_case()
    c1_run_case()
    densify_case()
    trainer_case()


if __name__ == "__main__":
    main()
