"""Learned prefetch end to end on a reduced out-of-core setup.

Traces of marched coarse nodes are logged by the renderer on random
fly-throughs, the network is trained on the GPU by libvt's kernels, and a
held-out spline fly-through is rendered from a cold cache with demand
paging alone and with the network's prefetch hints.  The images must be
identical frame by frame (a prediction never changes a pixel); the hints
must load bricks ahead of demand, raise the device-cache hit rate and cut
the demand requests and passes.  The device cache holds every brick of the
scene: each frame of this small scene touches most of its bricks, so a
smaller cache is refilled within every frame and leaves no slot that the
next frame's prefetch may take."""
import numpy as np
import pytest

import visualtur_b200 as vt
from visualtur_b200 import prefetch as pf

pytestmark = pytest.mark.gpu

N, ISO, LC, LO, LEVEL = 256, 0.6, 4, 6, 3
W, H, FOV = 96, 72, 30.0


@pytest.fixture(scope="module")
def scene(tmp_path_factory):
    d = tmp_path_factory.mktemp("pf")
    vol = vt.generate_volume(vt.VT_GEN_BLOBS, 17, (N, N, N), (48, 6.0, 24.0, 0.5, 1.5, 0.05))
    path = str(d / "blobs.oct")
    vt.build_octree(vt.FileManager.wrap(vol), ISO, path)
    return vol, path


def make(vol, path, dev_slots, host_slots, **opt):
    fm, oc = vt.FileManager.wrap(vol), vt.Octree(path)
    p = vt.make_params(W=W, H=H, octreeFile=None, hdf5File=None, octreeLevel=LO, levelCubes=LC, dimCube=16,
                       distance=50.0, fov_H=FOV, fov_W=FOV, maxElementsCache=dev_slots,
                       maxElementsCache_CPU=host_slots)
    return vt.visualTur(p, vt.default_options(**opt), volume=fm, octree=oc), (fm, oc)


def test_learned_prefetch_gains_over_demand_paging(scene, cuda):
    torch = cuda
    vol, path = scene
    # traces from random fly-throughs (resident renderer with the access log)
    tr, keep = make(vol, path, 8 ** LC, 8 ** LC, resident=1, record_trace=1, trace_level=LEVEL, record_hits=0)
    rng = np.random.default_rng(123)
    X, Y = [], []
    for path_i in range(20):
        pos, tgt = pf.random_flythrough(rng, N, 60, 1.2 * N, 1.8 * N)
        for p_, t_ in zip(pos, tgt):
            cam = pf.look_at(W, H, 50.0, FOV, p_, t_)
            tr.set_camera(cam)
            tr.render_host(rgb8=False)
            X.append(pf.pose_features(cam, N, FOV))
            Y.append(pf.trace_to_targets(tr.trace(LEVEL), LEVEL))
    X, Y = np.array(X), np.array(Y)
    assert 0.02 < Y.mean() < 0.9
    bricks = tr.brick_list()
    P = pf.Prefetcher(N, FOV, LC, bricks, seed=1, hidden=128, level=LEVEL)
    hist = P.train(torch, X, Y, epochs=40, batch=128, lr=2e-3)
    assert hist[-1] < 0.6 * hist[0]

    # held-out spline, cold start
    pos, tgt = pf.random_flythrough(np.random.default_rng(999), N, 60, 1.3 * N, 1.7 * N)
    cams = [pf.look_at(W, H, 50.0, FOV, p_, t_) for p_, t_ in zip(pos, tgt)]
    dev = len(bricks)
    results = {}
    for mode in ("demand", "learned"):
        r, keep2 = make(vol, path, dev, len(bricks), resident=0, preload=0, record_hits=0)
        imgs, passes = [], []
        if mode == "learned":
            r.prefetch(P.bricks_for(P.predict(torch, pf.pose_features(cams[0], N, FOV))[0], 0.3))
        for k, cam in enumerate(cams):
            if mode == "learned" and k + 1 < len(cams):
                probs = P.predict(torch, pf.pose_features(cams[k + 1], N, FOV))[0]
                r.prefetch_hint(P.bricks_for(probs, 0.3))
            r.set_camera(cam)
            rgba, _ = r.render_host(rgb8=False)
            imgs.append(rgba)
            passes.append(r.stats()["passes"])
        s = r.stats()
        hit_rate = s["device_hits"] / max(1, s["device_hits"] + s["device_misses"])
        results[mode] = dict(imgs=imgs, passes=np.mean(passes), hit_rate=hit_rate, stats=s)
        r.close()
    for a, b in zip(results["demand"]["imgs"], results["learned"]["imgs"]):
        assert np.array_equal(a, b)
    dem, lrn = results["demand"], results["learned"]
    assert lrn["stats"]["bricks_prefetched"] > 0
    assert lrn["hit_rate"] > dem["hit_rate"]
    assert lrn["stats"]["bricks_requested"] < dem["stats"]["bricks_requested"]
    assert lrn["passes"] < dem["passes"]


def test_baseline_network_gains_over_demand_paging(workdir, cuda):
    """The learned-prefetch configuration itself: the 12 -> 512 -> 512 ->
    4096 network over level-4 nodes, trained by libvt's kernels with BCE on
    20 000 (pose, marched-node set) pairs logged by the renderer on random
    fly-throughs of the 1024^3 blob volume, then judged on a held-out
    spline fly-through from a cold cache against demand paging alone: the
    same pixels in every frame, fewer demand misses and passes, a higher
    device hit rate.  Prediction runs on the device (vt_prefetch_predict):
    features, forward pass, threshold and the brick requests, with no
    synchronisation in the frame loop.  Stall times are printed."""
    import time

    import test_gpu_configs as TC
    torch = cuda
    wl = TC.workload("c2s", torch, workdir)
    cfg = TC.bench.CONFIGS["c2s"]
    n, fov, lc = cfg["n"], cfg["fov"], cfg["levelC"]
    # traces: a resident renderer logs the level-4 nodes each pose marches
    p = vt.make_params(W=240, H=135, octreeFile=None, hdf5File=None, octreeLevel=cfg["levelO"], levelCubes=lc,
                       dimCube=16, distance=cfg["dist"], fov_H=fov, fov_W=fov)
    tr = vt.visualTur(p, vt.default_options(resident=1, record_trace=1, trace_level=pf.TRACE_LEVEL, record_hits=0),
                      volume=wl.fm, octree=wl.oc)
    X, Y = pf.collect_traces(tr, n, 240, 135, fov, np.random.default_rng(7), 100, 200, 1250.0 * n / 1024, 1750.0 * n / 1024,
                             dist=cfg["dist"])
    bricks = tr.brick_list()
    tr.close()
    assert X.shape == (20000, 12) and Y.shape == (20000, 4096) and 0.01 < Y.mean() < 0.9
    P = pf.Prefetcher(n, fov, lc, bricks, seed=11)
    assert P.mlp.dims == (12, 512, 512, 4096)
    hist = P.train(torch, X, Y, epochs=30, batch=256, lr=1e-3)
    assert hist[-1] < 0.5 * hist[0]

    pos, tgt = pf.random_flythrough(np.random.default_rng(999), n, 120, 1300.0 * n / 1024, 1700.0 * n / 1024)
    cams = [pf.look_at(960, 540, cfg["dist"], fov, p_, t_) for p_, t_ in zip(pos, tgt)]
    stream = torch.cuda.Stream()
    res = {}
    for mode in ("demand", "learned"):
        r = vt.visualTur(wl.params(), vt.default_options(resident=0, preload=0, record_hits=0, persistent=1,
                                                         lookahead=0, spec_async=1), volume=wl.fm, octree=wl.oc)
        # frames rendered at 960x540 through batch views (the handle's own size is 1920x1080)
        out = torch.empty(960 * 540 * 4, dtype=torch.float32, device="cuda")
        imgs, stall, passes = [], 0.0, 0
        t0 = time.perf_counter()
        for k, cam in enumerate(cams):
            if mode == "learned":
                r.prefetch_predict(P.mlp, cams[k:k + 4], n, fov, 0.5, stream=stream.cuda_stream)
            v = vt.vt_view()
            v.cam, v.dev_rgba, v.dev_rgb8 = cam, out.data_ptr(), None
            r.render_batch([v], stream=stream.cuda_stream)
            s = r.stats()
            stall += s["ms_stall_last_frame"]
            passes += s["passes"]
            stream.synchronize()
            imgs.append(out.cpu().numpy().copy())
        wall = time.perf_counter() - t0
        s = r.stats()
        res[mode] = dict(imgs=imgs, stall=stall / len(cams), passes=passes / len(cams), wall=wall, stats=s,
                         hit=s["device_hits"] / max(1, s["device_hits"] + s["device_misses"]))
        r.close()
    for a, b in zip(res["demand"]["imgs"], res["learned"]["imgs"]):
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32))
    dem, lrn = res["demand"], res["learned"]
    print("\nlearned prefetch, held-out 120-frame spline at 960x540 (c2s volume, cold cache):")
    for k, v in res.items():
        print("  %-7s stall %.3f ms/frame, passes %.2f/frame, hit rate %.4f, device misses %d, bricks loaded %d, "
              "predicted %d, wall %.3f s" % (k, v["stall"], v["passes"], v["hit"], v["stats"]["device_misses"],
                                             v["stats"]["bricks_loaded_disk"], v["stats"]["bricks_hinted"], v["wall"]))
    assert lrn["stats"]["bricks_spec_loaded"] > 0
    assert lrn["hit"] > dem["hit"]
    assert lrn["stats"]["device_misses"] < dem["stats"]["device_misses"]
    assert lrn["passes"] < dem["passes"]
