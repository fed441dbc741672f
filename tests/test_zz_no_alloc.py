"""The ICP entry point that allocates nothing (of_icp_track_static).

Some callers cannot allocate device memory once they are running: hosts that
own every device allocation up front (plugin hosts with a fixed memory budget)
or real-time loops that cannot afford cudaMalloc's implicit synchronisation or
a failure in the middle of a session. For them of_icp_track_static takes no
workspace and uses a fixed device array inside the library instead. This test
calls it through the C-ABI on two frames in a row and checks that every result
equals the one of_icp_track gives with a caller-owned workspace: both run the
same kernel on the same grid with a fixed summation order, so the poses and
the whole statistics record (status, inliers, iterations, residual, smallest
pivot) must be identical bit for bit -- tighter than the parity tests' pose
tolerance (1e-5 rad, 0.01 mm), which the pose meets too. It runs last so that a
failure here cannot hide another test's result, and it builds all of its own
inputs so that it also passes alone in a fresh process.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _pose_error(P, G):
    R = P[:3, :3].T @ G[:3, :3]
    rot = float(np.arccos(np.clip((np.trace(R) - 1.0) / 2.0, -1.0, 1.0)))
    return rot, float(np.linalg.norm(P[:3, 3] - G[:3, 3]))


def test_static_workspace_matches_caller_workspace_on_two_calls():
    import torch

    import openfusion_b200 as of
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    dev = torch.device("cuda:0")
    cfg = of.CONFIGS["c1"]
    seq = of.make_sequence(cfg, frames=4)

    def pose_tensor(P):
        return torch.tensor(np.asarray(P, np.float64).reshape(16), dtype=torch.float64, device=dev)

    vol, lam = of.new_volume(cfg, dev), of.lambda_table(cfg, dev)
    for k in range(2):
        of.integrate(cfg, vol, torch.from_numpy(seq.depth[k].astype(np.int16)).to(dev),
                     pose_tensor(seq.poses[k]), lam)
    model = of.raycast(cfg, vol, pose_tensor(seq.poses[1]))
    lib = of._native.lib()
    stream = torch.cuda.current_stream().cuda_stream
    cam, icp = cfg.camera(), cfg.icp()

    pose_static = pose_tensor(seq.poses[1])
    pose_ref = pose_tensor(seq.poses[1])
    ws = of.icp_workspace(cfg, dev)
    for k in (2, 3):  # two calls in a row, each starting from the previous result
        frame = of.preprocess(cfg, torch.from_numpy(seq.depth[k].astype(np.int16)).to(dev))
        stats_static = torch.zeros(32, dtype=torch.uint8, device=dev)
        stats_ref = torch.zeros(32, dtype=torch.uint8, device=dev)
        st = lib.of_icp_track_static(C.byref(cam), C.byref(icp), frame.data_ptr(),
                                     model.data_ptr(), pose_static.data_ptr(),
                                     stats_static.data_ptr(), stream)
        assert st == 0, lib.of_status_string(st)
        of.icp_track(cfg, frame, model, pose_ref, ws, stats_ref)
        torch.cuda.synchronize()
        Ps = pose_static.cpu().numpy().reshape(4, 4)
        Pr = pose_ref.cpu().numpy().reshape(4, 4)
        rot, trans = _pose_error(Ps, Pr)
        assert rot < 1e-5 and trans < 1e-2, (k, rot, trans)
        assert np.array_equal(Ps, Pr), (k, Ps - Pr)
        ss = stats_static.cpu().numpy()
        sr = stats_ref.cpu().numpy()
        assert ss.view(np.int32)[0] == 0 and ss.view(np.int32)[2] > 0
        assert np.array_equal(ss, sr), (ss.view(np.int32)[:4], sr.view(np.int32)[:4],
                                        ss[16:].view(np.float64), sr[16:].view(np.float64))
        # and the tracked pose follows the ground truth of the frame
        rot_gt, trans_gt = _pose_error(Ps, seq.poses[k])
        assert rot_gt < np.radians(0.5) and trans_gt < 5.0
