"""Batched streams (of_batch_*): many independent streams, one launch per
stage, against the single-stream tracker on the same frames.

Per stream, pre-processing, integration and the raycast of a batch write
exactly what the single-stream stages write (bit for bit); the batched ICP
sums in another order, so poses agree within the pose tolerance. The tuning
knobs change no result, so a tuned batch equals an untuned one bit for bit,
and a batch replayed as CUDA graphs equals the eager one.
"""
import ctypes as C
import dataclasses

import numpy as np
import pytest

from conftest import pose_error

pytestmark = pytest.mark.gpu


def mixed_configs(of):
    """Five small streams of different resolution, volume and cube size."""
    base = of.c4_configs(count=5, seed=4100, frames=8)
    shapes = [((160, 120), 128, 2000.0), ((320, 240), 128, 2500.0), ((160, 120), 256, 3000.0),
              ((320, 240), 256, 2200.0), ((640, 480), 128, 2800.0)]
    out = []
    for c, ((w, h), res, size) in zip(base, shapes):
        f = 525.0 * w / 640.0
        out.append(dataclasses.replace(c, width=w, height=h, fx=f, fy=f, cx=(w - 1) / 2.0,
                                       cy=(h - 1) / 2.0, resolution=res, size_mm=size,
                                       trunc_mm=max(30.0, 4.0 * size / res)))
    return out


def sequences(of, cfgs, frames, cuda):
    import torch
    seqs = [of.make_sequence(c, frames=frames) for c in cfgs]
    depth = [[torch.from_numpy(s.depth[k].astype(np.int16)).to(cuda) for s in seqs]
             for k in range(frames)]
    return seqs, depth


def export_volume(of, cfg, vol_ptr, cuda):
    import torch
    m = cfg.resolution ** 3
    tsdf = torch.empty(m, dtype=torch.float32, device=cuda)
    wgt = torch.empty(m, dtype=torch.int16, device=cuda)
    st = torch.cuda.current_stream().cuda_stream
    assert of._native.lib().of_volume_export(C.byref(cfg.volume()), C.c_void_p(vol_ptr),
                                             tsdf.data_ptr(), wgt.data_ptr(), st) == 0
    torch.cuda.synchronize()
    return tsdf.cpu().numpy(), wgt.cpu().numpy()


def level0_points(of, cfg, pyr_ptr, cuda):
    import torch
    n = cfg.width * cfg.height
    v = torch.empty(3 * n, dtype=torch.float32, device=cuda)
    nn = torch.empty(3 * n, dtype=torch.float32, device=cuda)
    st = torch.cuda.current_stream().cuda_stream
    assert of._native.lib().of_points_to_reference(C.byref(cfg.camera()), C.c_void_p(pyr_ptr),
                                                   None, v.data_ptr(), nn.data_ptr(), st) == 0
    torch.cuda.synchronize()
    return v.cpu().numpy(), nn.cpu().numpy()


def test_batched_stages_equal_single_stream_stages(of, cuda):
    """After two steps every stream's volume (frame 0 fused), model (raycast
    at pose 0) and frame maps (frame 1) equal the single-stream tracker's
    bit for bit; the tracked poses agree within 1e-5 rad / 0.01 mm."""
    cfgs = mixed_configs(of)
    seqs, depth = sequences(of, cfgs, 2, cuda)
    batch = of.Batch(cfgs, [s.poses[0] for s in seqs])
    for k in range(2):
        batch.process(depth[k])
    P = batch.poses()
    for i, c in enumerate(cfgs):
        tr = of.Tracker(c, seqs[i].poses[0])
        for k in range(2):
            tr.process(depth[k][i])
        Pt = tr.pose_history(2)[1]
        tb, bb = tr.buffers(), batch.buffers(i)
        t1, w1 = export_volume(of, c, tb.volume, cuda)
        t2, w2 = export_volume(of, c, bb.volume, cuda)
        assert np.array_equal(w1, w2) and np.array_equal(t1, t2), c.name
        for a, b in ((tb.model, bb.model), (tb.frame, bb.frame)):
            v1, n1 = level0_points(of, c, a, cuda)
            v2, n2 = level0_points(of, c, b, cuda)
            assert np.array_equal(v1, v2) and np.array_equal(n1, n2), c.name
        rot, trans = pose_error(P[i], Pt)
        assert rot < 1e-5 and trans < 1e-2, (c.name, rot, trans)
        tr.close()
    batch.close()


def test_batch_tracks_every_stream(of, cuda):
    """Eight frames of five mixed streams: every stream stays on its ground
    truth, and the poses agree with the single-stream trackers'."""
    cfgs = mixed_configs(of)
    n = 8
    seqs, depth = sequences(of, cfgs, n, cuda)
    batch = of.Batch(cfgs, [s.poses[0] for s in seqs])
    hist = []
    for k in range(n):
        batch.process(depth[k])
        P, stats = batch.poses(with_stats=True)
        hist.append(P)
        if k > 0:
            assert all(s.status == 0 for s in stats)
    batch.close()
    for i, c in enumerate(cfgs):
        tr = of.Tracker(c, seqs[i].poses[0])
        for k in range(n):
            tr.process(depth[k][i])
        ht = tr.pose_history(n)
        tr.close()
        for k in range(n):
            r_gt, t_gt = pose_error(hist[k][i], seqs[i].poses[k])
            assert r_gt < np.radians(1.0) and t_gt < 20.0, (c.name, k, r_gt, t_gt)
            rot, trans = pose_error(hist[k][i], ht[k])
            assert rot < 1e-4 and trans < 0.1, (c.name, k, rot, trans)


def test_tuned_and_graph_batches_equal_the_eager_one(of, cuda):
    """Online tuning (every knob's candidates timed on the first steps) and
    graph replay change no result: poses and a volume equal bit for bit."""
    cfgs = mixed_configs(of)[:4]
    n = 40  # > the tuning steps (7 + 5 + up to 3 candidates, twice each)
    seqs, depth = sequences(of, cfgs, n, cuda)
    runs = []
    for graph, tune in ((False, False), (True, True), (True, False)):
        batch = of.Batch(cfgs, [s.poses[0] for s in seqs], use_graph=graph, tune=tune)
        hist = []
        for k in range(n):
            batch.process(depth[k])
            hist.append(batch.poses())
        batch.flush()
        t, w = export_volume(of, cfgs[1], batch.buffers(1).volume, cuda)
        tun = batch.tuning()
        runs.append((np.array(hist), t, w, (tun.ray_tile, tun.list_div, tun.icp_clusters, tun.tuned)))
        batch.close()
    assert runs[1][3][3] == 1, runs[1][3]
    assert 0 <= runs[1][3][0] < 7 and 0 <= runs[1][3][1] < 5 and runs[1][3][2] >= 1
    for r in runs[1:]:
        assert np.array_equal(r[0], runs[0][0])
        assert np.array_equal(r[1], runs[0][1]) and np.array_equal(r[2], runs[0][2])


def all_shapes_configs(of):
    """Six streams covering every resolution {160x120, 320x240, 640x480} and
    every volume {128^3, 256^3, 512^3} of the batched-streams workload."""
    base = of.c4_configs(count=6, seed=4300, frames=4)
    shapes = [((160, 120), 128, 2000.0), ((320, 240), 256, 2500.0), ((640, 480), 512, 3000.0),
              ((160, 120), 512, 2400.0), ((640, 480), 128, 2800.0), ((320, 240), 512, 2200.0)]
    out = []
    for c, ((w, h), res, size) in zip(base, shapes):
        f = 525.0 * w / 640.0
        out.append(dataclasses.replace(c, width=w, height=h, fx=f, fy=f, cx=(w - 1) / 2.0,
                                       cy=(h - 1) / 2.0, resolution=res, size_mm=size,
                                       trunc_mm=max(30.0, 4.0 * size / res)))
    return out


def test_batched_icp_matches_oracle_per_stream(of, ora, cuda):
    """Stepwise parity of the batched ICP (k_icp_batch) at the pose
    tolerance (1e-5 rad, 0.01 mm): after the third step of a batch of six
    streams of every resolution and volume, each stream's pose equals the FP64
    oracle's multi-level ICP (10/5/4 iterations) run on that stream's own
    frame and model pyramids from the pose it started the step at."""
    import torch
    from test_gpu_parity import gpu_pyramid_to_oracle
    cfgs = all_shapes_configs(of)
    seqs, depth = sequences(of, cfgs, 3, cuda)
    batch = of.Batch(cfgs, [s.poses[0] for s in seqs])
    for k in range(2):
        batch.process(depth[k])
    start = batch.poses()
    batch.process(depth[2])
    P, stats = batch.poses(with_stats=True)
    for i, c in enumerate(cfgs):
        b = batch.buffers(i)
        frame = of.copy_pyramid(c, b.frame, cuda)
        model = of.copy_pyramid(c, b.model, cuda)
        torch.cuda.synchronize()
        fbuf, _ = gpu_pyramid_to_oracle(of, ora, c, frame)
        mbuf, _ = gpu_pyramid_to_oracle(of, ora, c, model, with_depth=False)
        st, opose, its = ora.icp_track(c, fbuf, mbuf, start[i])
        assert st == 0 and stats[i].status == 0, (c.name, st, stats[i].status)
        assert stats[i].iterations == its == sum(c.iters), (c.name, stats[i].iterations, its)
        rot, trans = pose_error(P[i], opose)
        assert rot < 1e-5 and trans < 1e-2, (c.name, rot, trans)
        rot_gt, trans_gt = pose_error(P[i], seqs[i].poses[2])
        assert rot_gt < np.radians(1.0) and trans_gt < 20.0, (c.name, rot_gt, trans_gt)
    batch.close()
