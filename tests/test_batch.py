"""Batched multi-scene training (u3dg_batch_*): every scene of a batch trains exactly as the same scene
trained alone, with or without the autotuner of tile size and compositing schedule, at tile 16 and at
tile 32 (four backward CTAs per tile with separate partial slots: deterministic)."""
from __future__ import annotations

import dataclasses

import numpy as np
import pytest

from univeral_3d_reconstruction_system_b200.scenes import PRESETS, make_scene
from univeral_3d_reconstruction_system_b200.types import RasterSettings, TrainImage

pytestmark = pytest.mark.gpu


def _scenes(u3dg):
    specs = [dataclasses.replace(PRESETS["tiny"], gt_count=1500, views=6),
             dataclasses.replace(PRESETS["small"], gt_count=6000, views=9, width=128, height=96, focal=120.0),
             dataclasses.replace(PRESETS["tiny"], gt_count=3000, views=5, width=112, height=80, focal=100.0)]
    out = []
    for k, sp in enumerate(specs):
        sc = make_scene(sp, 40 + k)
        imgs = u3dg.renderViewsSh(sc.truth, sc.sh_rest, 3, sc.cameras, RasterSettings())
        sc.images = [TrainImage(c, im) for c, im in zip(sc.cameras, imgs)]
        init = u3dg.initGaussiansFromPoints(sc.init_xyz, sc.init_rgb)
        out.append((init, sc.images, sc.extent, sc.options()))
    return out


def _alone(u3dg, scene, tile, raster, iterations):
    init, imgs, extent, opt = scene
    opt = dataclasses.replace(opt, raster=dataclasses.replace(opt.raster, tile_size=tile))
    t = u3dg.Trainer(init, imgs, extent, opt)
    t.set_raster_schedule(*raster)
    t.step(iterations)
    return t.model().flat(), t.stats()


@pytest.mark.parametrize("autotune,tile", [(False, 16), (False, 32), (True, 0)])
def test_batch_matches_scenes_trained_alone(u3dg, autotune, tile):
    scenes = _scenes(u3dg)
    if tile:
        scenes = [(i, im, e, dataclasses.replace(o, raster=dataclasses.replace(o.raster, tile_size=tile)))
                  for i, im, e, o in scenes]
    b = u3dg.Batch(scenes, autotune=autotune)
    assert len(b) == 3
    b.step(77)
    ms = b.time_steps(50)
    assert ms > 0
    b.step(123)  # past every scene's refine_stop: rounds of all scenes as one graph launch
    launches, captures = b.graph_launches()
    assert launches >= 3 and 1 <= captures <= launches
    for k, scene in enumerate(scenes):
        tile, tuned = b.tile_size(k)
        tile2, raster, tuned2 = b.schedule(k)
        assert (tile2, tuned2) == (tile, tuned)
        assert tile in (8, 16, 32) and raster[0] in (8, 16) and raster[1] in (1, 2) and raster[2] in (1, 2)
        if not autotune:
            assert (tile, raster, tuned) == (scene[3].raster.tile_size, (8, 1, 1), 0.0)
        else:
            assert tuned > 0
        t = b.trainer(k)
        assert t.iteration() == 250
        flat, st = _alone(u3dg, scene, tile, raster, 250)
        np.testing.assert_array_equal(t.model().flat(), flat)
        s2 = t.stats()
        assert (s2.iteration, s2.loss, s2.psnr, s2.gaussians) == (st.iteration, st.loss, st.psnr, st.gaussians)
    b.close()
