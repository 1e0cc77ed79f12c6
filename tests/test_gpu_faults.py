"""Bounded waits and host-side failures at render time, forced with small
bounds or a failing volume reader (no GPU fault is caused: every failure is
made on the host or by a bounded host loop).  Each test checks the status,
that the message says what happened, and that the same renderer then
renders a frame equal to the oracle's -- a failed frame leaves no brick
stuck in the requested state.

Reference behaviour this replaces: HDF5 errors exit(0)
(src/FileManager.cu:15-36); per-pass cache admission defers rays
(src/lruCache.cu:184-192); the iterate-until-PAINTED loop has no bound
(src/visualTur.cu:167-228)."""
import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc
from test_gpu_parity import assert_parity, oracle_render

pytestmark = pytest.mark.gpu


def make(case, workdir, fm=None, dev=None, host=None, **opt):
    c = F.CASES[case]
    vol = F.case_volume(case)
    fm = fm if fm is not None else vt.FileManager.wrap(vol)
    oc = vt.Octree(F.case_octree(case, workdir))
    nb = 8 ** c["levelC"]
    p = vt.make_params(W=c["W"], H=c["H"], octreeFile=None, hdf5File=None, octreeLevel=c["levelO"],
                       levelCubes=c["levelC"], dimCube=1 << (int(np.log2(c["n"])) - c["levelC"]),
                       cubeInc=c["inc"], distance=c["dist"], fov_H=c["fov"], fov_W=c["fov"],
                       maxElementsCache=dev or nb, maxElementsCache_CPU=host or nb)
    o = dict(resident=0, preload=0, record_hits=1)
    o.update(opt)
    r = vt.visualTur(p, vt.default_options(**o), volume=fm, octree=oc)
    m = {"mv": r.camera_Move, "rx": r.camera_RotateX, "ry": r.camera_RotateY, "rz": r.camera_RotateZ,
         "mf": r.camera_MoveForward, "mu": r.camera_MoveUpward, "sr": r.camera_StrafeRight}
    for op, v in c["ops"]:
        m[op](v)
    return r


def frame(r):
    rgba, rgb8 = r.render_host()
    node, brick, t, nrm = r.debug_hits()
    return dict(rgba=rgba, rgb8=rgb8, node=node, brick=brick, t=t, normal=nrm, stats=r.stats())


def test_pass_bound_times_out_and_later_frames_finish(workdir, cuda):
    """max_passes = 2 on a cold cache: the frame needs more passes and
    returns VT_ERR_TIMEOUT; the bricks its passes loaded stay, so repeating
    the frame makes progress until it completes, equal to the oracle."""
    free = frame(make("c1", workdir, lookahead=0, skip=0))
    assert free["stats"]["passes"] >= 3          # the cold frame needs more than the bound
    r = make("c1", workdir, max_passes=2, lookahead=0, skip=0)
    with pytest.raises(vt.VtError) as e:
        r.render_host()
    assert e.value.status == vt.VT_ERR_TIMEOUT and "max_passes" in str(e.value)
    for attempt in range(64):
        try:
            got = frame(r)
            break
        except vt.VtError as err:
            assert err.status == vt.VT_ERR_TIMEOUT
    else:
        pytest.fail("the frame never completed")
    assert_parity(got, oracle_render("c1", workdir))
    r.close()


@pytest.mark.parametrize("persistent", [0, 1])
def test_request_list_bound_defers_requests_to_later_passes(persistent, workdir, cuda):
    """At most 3 brick requests a pass: the rest wait for the next pass
    (counted in requests_deferred); the image is unchanged."""
    free = frame(make("c1", workdir, persistent=persistent))
    r = make("c1", workdir, persistent=persistent, max_requests=3, lookahead=2)
    got = frame(r)
    st = got["stats"]
    assert st["requests_deferred"] > 0
    assert st["passes"] > free["stats"]["passes"]
    assert_parity(got, oracle_render("c1", workdir))
    r.close()


def test_suspended_list_bound_fails_the_frame_cleanly(workdir, cuda):
    """Room for 8 waiting rays: a cold frame overflows and returns
    VT_ERR_STATE; with every brick loaded the same renderer's frame needs
    no waiting and equals the oracle."""
    r = make("s64", workdir, max_suspended=8)
    with pytest.raises(vt.VtError) as e:
        r.render_host()
    assert e.value.status == vt.VT_ERR_STATE and "suspended-ray list overflow" in str(e.value)
    assert r.prefetch(r.brick_list()) > 0
    got = frame(r)
    assert got["stats"]["passes"] == 1
    assert_parity(got, oracle_render("s64", workdir))
    r.close()


@pytest.mark.parametrize("mode", ["demand", "demand_skip", "persist_skip"])
def test_stack_pool_overflow_restarts_rays_with_the_same_pixels(mode, workdir, cuda):
    """One pool entry per ray: most suspended rays cannot save their stack
    and restart from the root next pass.  Pixels, hit nodes and the hit
    count still equal the oracle's (a tentative hit dropped with the pool is
    found again and counted once)."""
    skip = 0 if mode == "demand" else 3
    r = make("c1", workdir, dev=40, host=40, pool_per_ray=1, skip=skip, lookahead=1,
             persistent=1 if mode.startswith("persist") else 0, pops=5)
    got = frame(r)
    want = oracle_render("c1", workdir)
    assert_parity(got, want)
    assert got["stats"]["hits"] == want["agg"]["hits"]
    assert got["stats"]["passes"] > 1
    r.close()


def test_failed_brick_reads_fail_the_frame_and_the_renderer_recovers(workdir, cuda):
    """The volume is read through a function that fails while `broken` is
    set (a short read or a missing brick file): the frame returns VT_ERR_IO
    with a message; once reads work again the same renderer renders the
    frame, equal to the oracle."""
    vol = F.case_volume("s64")
    state = {"broken": True, "calls": 0}

    def read(s, e):
        state["calls"] += 1
        if state["broken"] and state["calls"] % 3 == 0:
            return None
        return orc.read_voxels(vol, s, e)
    fm = vt.FileManager.from_reader(read, vol.shape)
    r = make("s64", workdir, fm=fm, dev=96, host=96)
    with pytest.raises(vt.VtError) as e:
        r.render_host()
    assert e.value.status == vt.VT_ERR_IO and "failed" in str(e.value)
    state["broken"] = False
    got = frame(r)
    assert_parity(got, oracle_render("s64", workdir))
    r.close()
