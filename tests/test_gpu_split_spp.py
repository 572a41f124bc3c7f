"""One frame's samples split over several renders (the data path of a frame
split over GPUs, minus the all-reduce that tests/test_shard_dist.py runs on
gloo ranks): renders of samples [f, f + n) with first_sample = f, summed,
equal one render of the whole frame, because each path's random stream is
keyed by the frame's sample index and the renders add radiance in 2^-32
fixed point. Only the float32 rounding of the per-ray sums handed out
separates the two."""
import numpy as np
import pytest

import hptracing_b200 as H
from hptracing_b200 import shard
from tests import scenes as S

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def room(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    mesh, nodes, leaf = S.make_scene(0)
    return H.Scene(mesh, nodes, leaf)


@pytest.fixture(scope="module")
def spheres(built):
    if H.device_count() == 0:
        pytest.skip("no CUDA device")
    mesh, nodes, leaf = S.make_scene(1, seed=1, texture_size=128)
    return H.Scene(mesh, nodes, leaf)


def _params(w, h, spp, depth, bg, first=0):
    return H.make_params(w, h, 1, 1, bg, spp, depth, 0, 1.0, 17, first_sample=first)


def _same_sums(a, b):
    """Per-ray float32 sums of the same fixed-point radiance, rounded at
    different points: equal non-finite markers, finite values within a few
    float32 ulps."""
    fa, fb = np.isfinite(a), np.isfinite(b)
    assert np.array_equal(fa, fb)
    assert np.array_equal(a[~fa], b[~fb], equal_nan=True)
    assert np.allclose(a[fa], b[fb], rtol=1e-6, atol=1e-6)


@pytest.mark.parametrize("scene_name,w,h,spp,depth,bg,world", [
    ("room", 64, 48, 8, 5, (0.0, 0.0, 0.0), 2),
    ("room", 64, 48, 8, 5, (0.2, 0.3, 0.4), 3),
    ("spheres", 64, 64, 6, 8, (0.1, 0.1, 0.1), 4),
])
def test_slices_sum_to_the_whole_frame(request, scene_name, w, h, spp, depth, bg, world):
    gpu = request.getfixturevalue(scene_name)
    cam = S.hp_camera(S.ROOM_CAM)
    whole_rgba, whole = gpu.render(cam, _params(w, h, spp, depth, bg), want_accum=True)
    total = np.zeros_like(whole)
    for first, count in shard.spp_slices(spp, world):
        if count:
            total += gpu.render(cam, _params(w, h, count, depth, bg, first), want_accum=True)[1]
    _same_sums(total, whole)
    # The image resolved from the summed accumulator: the whole render's up
    # to the float32 rounding of the sums (at most one step of 255).
    rgba = H.resolve(total, w, h, 1, 1, spp)
    diff = np.abs(rgba.astype(np.int16) - whole_rgba.astype(np.int16))
    assert diff.max() <= 1
    assert (diff == 0).mean() > 0.999


def test_render_split_spp_single_rank(room):
    """The library entry point on one rank: the whole frame's accumulator
    and image."""
    cam = S.hp_camera(S.ROOM_CAM)
    p = _params(48, 40, 6, 5, (0.1, 0.1, 0.1))
    whole_rgba, whole = room.render(cam, p, want_accum=True)
    rgba, acc = shard.render_split_spp(room, cam, p, rank=0, world=1)
    _same_sums(acc, whole)
    assert np.abs(rgba.astype(np.int16) - whole_rgba.astype(np.int16)).max() <= 1


def test_first_sample_selects_the_random_streams(room):
    """Samples [3, 8) are not samples [0, 5): first_sample moves the random
    streams; and an invalid first_sample is rejected."""
    cam = S.hp_camera(S.ROOM_CAM)
    a = room.render(cam, _params(32, 24, 5, 5, (0, 0, 0), 0), want_accum=True)[1]
    b = room.render(cam, _params(32, 24, 5, 5, (0, 0, 0), 3), want_accum=True)[1]
    c = room.render(cam, _params(32, 24, 5, 5, (0, 0, 0), 3), want_accum=True)[1]
    assert not np.array_equal(a, b)
    assert np.array_equal(b, c, equal_nan=True)
    with pytest.raises(H.HptError):
        room.render(cam, _params(32, 24, 5, 5, (0, 0, 0), -1))
