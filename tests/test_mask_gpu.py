"""Pixel-mask stamping (sf_engine_set_pixel_mask): the detector's pixel mask
written into the frames as the masked sentinel before the threshold. The
reference reads no pixel mask; the check is that a masked run equals the
oracle's dext (src/dext.cc) on the frame with the mask stamped in by hand,
and that clearing the mask (and replaying captured graphs) restores the
unmasked result."""

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("dtype", [np.uint16, np.uint32])
def test_mask_matches_stamped_frames(gpu_lib, dtype):
    from dials_metal_spotfinder_b200 import synth
    from dials_metal_spotfinder_b200.engine import Engine
    rng = np.random.default_rng(21)
    a = synth.eiger_4m(frames=1).frame(0).astype(dtype)
    b = rng.poisson(2.0, (300, 517)).astype(dtype)
    b[rng.random(b.shape) < 0.004] = 3000
    frames = [a, b]
    masks = []
    for img in frames:
        m = rng.random(img.shape) < 0.01
        m[40:60, 100:180] = True           # a dead region
        m[:, img.shape[1] // 2] = True     # a bad column
        masks.append(m)
    maxval = np.iinfo(dtype).max
    with Engine([f.shape for f in frames], dtype, slots=2) as eng:
        eng.use_graph(True)
        for s in range(2):
            for f, img in enumerate(frames):
                eng.upload(s, f, img)
        eng.run(0)  # a graph captured without a mask
        eng.synchronize()
        for f, m in enumerate(masks):
            eng.set_pixel_mask(f, m)
        eng.run(1)
        eng.synchronize()
        for f, (img, m) in enumerate(zip(frames, masks)):
            stamped = img.copy()
            stamped[m] = maxval
            assert eng.signal(1, f).tobytes() == O.dext(stamped)[1].tobytes(), f
        eng.set_pixel_mask(0, None)
        for f, img in enumerate(frames):
            eng.upload(0, f, img)
        eng.run(0)
        eng.synchronize()
        assert eng.signal(0, 0).tobytes() == O.dext(frames[0])[1].tobytes()
        stamped = frames[1].copy()
        stamped[masks[1]] = maxval
        assert eng.signal(0, 1).tobytes() == O.dext(stamped)[1].tobytes()
