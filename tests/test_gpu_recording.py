"""A recording as the tracker's frame source (of_reader_*): the prefetching
reader delivers every frame bit for bit, ends with OF_END_OF_SEQUENCE, and a
tracker fed from it tracks exactly as one fed from device memory."""
import dataclasses

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("prefetch", [1, 4])
def test_reader_feeds_the_tracker(of, cuda, tmp_path, prefetch):
    import torch
    cfg = dataclasses.replace(of.CONFIGS["c1"])
    n = 10
    seq = of.make_sequence(cfg, frames=n)
    of.write_recording(tmp_path, cfg, seq.depth.astype(np.uint16))
    rd = of.Reader(tmp_path, prefetch=prefetch)
    assert (rd.width, rd.height, rd.frames) == (cfg.width, cfg.height, n)
    tr_file = of.Tracker(cfg, seq.poses[0])
    buf = torch.empty((cfg.height, cfg.width), dtype=torch.int16, device=cuda)
    for k in range(n):
        d = rd.next(buf)
        assert d is not None
        torch.cuda.synchronize()
        assert np.array_equal(d.cpu().numpy().view(np.uint16), seq.depth[k].astype(np.uint16))
        tr_file.process(d)
    assert rd.next(buf) is None
    rd.close()
    tr_mem = of.Tracker(cfg, seq.poses[0])
    for k in range(n):
        tr_mem.process(torch.from_numpy(seq.depth[k].astype(np.int16)).to(cuda))
    assert np.array_equal(tr_file.pose_history(n), tr_mem.pose_history(n))
    tr_file.close()
    tr_mem.close()
