"""ctypes binding of the CPU oracle (liboracle.so).

TEST INFRASTRUCTURE ONLY: a literal host restatement of the reference's
algorithm (see vt_oracle.h).  Imported by tests/, __graft_entry__.smoke()
and bench.py's CPU-baseline / reference legs as the checker; the product in
visualtur_b200/ never imports it.
"""
import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")


def build(force=False):
    src = [os.path.join(HERE, f) for f in ("vt_oracle.cpp", "vt_oracle.h", "Makefile")]
    if force or not os.path.exists(LIB_PATH) or any(os.path.getmtime(s) > os.path.getmtime(LIB_PATH) for s in src):
        subprocess.run(["make", "-C", HERE, "-B" if force else "all"], check=True, capture_output=True)
    return LIB_PATH


class orc_f3(C.Structure):
    _fields_ = [("x", C.c_float), ("y", C.c_float), ("z", C.c_float)]


class orc_camera(C.Structure):
    _fields_ = [("H", C.c_int), ("W", C.c_int), ("numRayPixel", C.c_int), ("distance", C.c_float),
                ("fov_h", C.c_float), ("fov_w", C.c_float), ("h", C.c_float), ("w", C.c_float),
                ("look", orc_f3), ("up", orc_f3), ("right", orc_f3), ("position", orc_f3),
                ("rotX", C.c_float), ("rotY", C.c_float), ("rotZ", C.c_float)]


class orc_render_params(C.Structure):
    _fields_ = [("levelO", C.c_int), ("levelC", C.c_int), ("cubeInc", C.c_int), ("iso", C.c_float),
                ("light", orc_f3), ("nthreads", C.c_int), ("ray_begin", C.c_int), ("ray_end", C.c_int),
                ("ray_stride", C.c_int), ("dirs", C.c_void_p), ("refine", C.c_int)]


class orc_render_out(C.Structure):
    _fields_ = [("node_id", C.c_void_p), ("brick_id", C.c_void_p), ("t", C.c_void_p), ("normal", C.c_void_p),
                ("rgba", C.c_void_p), ("rgb8", C.c_void_p)] + \
               [(n, C.c_int64) for n in ("rays", "hits", "samples", "normal_samples", "candidates", "expansions",
                                         "max_stack", "stack_overflow_rays", "oob_taps")]


_P = C.c_void_p
_I3 = C.c_int * 3
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        L = C.CDLL(LIB_PATH)
        cam = C.POINTER(orc_camera)
        protos = {
            "orc_camera_init": (None, [cam, C.c_int, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]),
            "orc_camera_move": (None, [cam, orc_f3]),
            "orc_camera_rotate_x": (None, [cam, C.c_float]),
            "orc_camera_rotate_y": (None, [cam, C.c_float]),
            "orc_camera_rotate_z": (None, [cam, C.c_float]),
            "orc_camera_move_forward": (None, [cam, C.c_float]),
            "orc_camera_move_upward": (None, [cam, C.c_float]),
            "orc_camera_strafe_right": (None, [cam, C.c_float]),
            "orc_camera_change_screen": (None, [cam, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]),
            "orc_camera_rays": (None, [cam, _P]),
            "orc_coordinate_to_index": (C.c_uint64, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_index_level": (C.c_int, [C.c_uint64]),
            "orc_min_box": (None, [C.c_uint64, C.c_int, C.c_int, _I3]),
            "orc_octree_load": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
            "orc_octree_free": (None, [_P]),
            "orc_octree_info": (None, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int), _I3, C.POINTER(C.c_int)]),
            "orc_octree_level_size": (C.c_int, [_P, C.c_int]),
            "orc_octree_level": (_P, [_P, C.c_int]),
            "orc_children_mask": (C.c_int, [_P, C.c_int, C.c_uint64]),
            "orc_render_frame": (C.c_int, [_P, _P, C.c_int, _I3, cam, C.POINTER(orc_render_params),
                                           C.POINTER(orc_render_out)]),
            "orc_render_cube": (None, [cam, _P, _I3, _I3, _I3, C.c_float, orc_f3, _P, C.POINTER(C.c_int64)]),
            "orc_read_voxels": (None, [_P, _I3, _I3, _I3, _P]),
            "orc_build_octree": (C.c_int, [_P, C.c_int, _I3, C.c_float, C.c_char_p]),
            "orc_lru_create": (_P, [C.c_int, C.c_int, C.c_int, C.c_int]),
            "orc_lru_free": (None, [_P]),
            "orc_lru_update": (C.c_int, [_P, C.c_int, _P, _P, _P, _P, _P]),
            "orc_lru_stats": (None, [_P, C.c_int64 * 5]),
        }
        for name, (res, args) in protos.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


class Camera:
    """Camera + Screen of the reference (src/Camera.cu, src/Screen.cpp)."""

    def __init__(self, H, W, distance, fov_H, fov_W):
        self.c = orc_camera()
        lib().orc_camera_init(C.byref(self.c), 1, H, W, distance, fov_H, fov_W)

    def Move(self, d):
        lib().orc_camera_move(C.byref(self.c), orc_f3(*d))

    def RotateX(self, a):
        lib().orc_camera_rotate_x(C.byref(self.c), a)

    def RotateY(self, a):
        lib().orc_camera_rotate_y(C.byref(self.c), a)

    def RotateZ(self, a):
        lib().orc_camera_rotate_z(C.byref(self.c), a)

    def MoveForward(self, d):
        lib().orc_camera_move_forward(C.byref(self.c), d)

    def MoveUpward(self, d):
        lib().orc_camera_move_upward(C.byref(self.c), d)

    def StrafeRight(self, d):
        lib().orc_camera_strafe_right(C.byref(self.c), d)

    def change_screen(self, W, H, fovW, fovH, d):
        lib().orc_camera_change_screen(C.byref(self.c), W, H, fovW, fovH, d)

    def rays(self):
        out = np.empty((self.c.W * self.c.H, 3), np.float32)
        lib().orc_camera_rays(C.byref(self.c), out.ctypes.data)
        return out

    def state(self):
        c = self.c
        f = lambda v: (v.x, v.y, v.z)
        return {"look": f(c.look), "up": f(c.up), "right": f(c.right), "position": f(c.position),
                "h": c.h, "w": c.w}


def apply_ops(cam, ops):
    """ops: list like [("mv", (x,y,z)), ("rx", a), ("mf", d), ...]."""
    for op, v in ops:
        {"mv": cam.Move, "rx": cam.RotateX, "ry": cam.RotateY, "rz": cam.RotateZ, "mf": cam.MoveForward,
         "mu": cam.MoveUpward, "sr": cam.StrafeRight}[op](v)


class Octree:
    def __init__(self, path):
        self._h = C.c_void_p()
        r = lib().orc_octree_load(path.encode(), C.byref(self._h))
        if r != 0:
            raise IOError("oracle: cannot load octree %s (%d)" % (path, r))
        iso, dim, nl = C.c_float(), C.c_int(), C.c_int()
        rd = _I3()
        lib().orc_octree_info(self._h, C.byref(iso), C.byref(dim), rd, C.byref(nl))
        self.iso, self.dimension, self.nLevels, self.realDim = iso.value, dim.value, nl.value, tuple(rd)

    def level(self, l):
        n = lib().orc_octree_level_size(self._h, l)
        if n <= 0:
            return np.zeros(0, np.uint64)
        p = lib().orc_octree_level(self._h, l)
        return np.ctypeslib.as_array(C.cast(p, C.POINTER(C.c_uint64)), (n,)).copy()

    def __del__(self):
        try:
            lib().orc_octree_free(self._h)
        except Exception:
            pass


def render(octree, volume, cam, levelO, levelC, cubeInc=3, iso=None, light=(0.0, 512.0, 0.0), nthreads=0,
           ray_begin=0, ray_end=0, ray_stride=1, dirs=None, refine=0):
    """Renders one frame; returns per-ray arrays and aggregate counters."""
    vol = np.ascontiguousarray(volume)
    vtype = 1 if vol.dtype == np.uint8 else 0
    n = cam.c.W * cam.c.H
    node = np.zeros(n, np.uint64)
    brick = np.zeros(n, np.uint64)
    t = np.full(n, -1.0, np.float32)
    nrm = np.zeros((n, 3), np.float32)
    rgba = np.ones((n, 4), np.float32)
    rgb8 = np.full((n, 3), 255, np.uint8)
    p = orc_render_params()
    p.levelO, p.levelC, p.cubeInc = levelO, levelC, cubeInc
    p.iso = octree.iso if iso is None else iso
    p.light = orc_f3(*light)
    p.nthreads, p.ray_begin, p.ray_end, p.ray_stride = nthreads, ray_begin, ray_end, ray_stride
    p.refine = refine
    d = None
    if dirs is not None:
        d = np.ascontiguousarray(dirs, np.float32)
        p.dirs = d.ctypes.data
    o = orc_render_out()
    o.node_id, o.brick_id, o.t = node.ctypes.data, brick.ctypes.data, t.ctypes.data
    o.normal, o.rgba, o.rgb8 = nrm.ctypes.data, rgba.ctypes.data, rgb8.ctypes.data
    r = lib().orc_render_frame(octree._h, vol.ctypes.data, vtype, _I3(*vol.shape), C.byref(cam.c), C.byref(p),
                               C.byref(o))
    if r != 0:
        raise ValueError("oracle render failed (%d)" % r)
    agg = {k: getattr(o, k) for k in ("rays", "hits", "samples", "normal_samples", "candidates", "expansions",
                                      "max_stack", "stack_overflow_rays", "oob_taps")}
    return {"node": node, "brick": brick, "t": t, "normal": nrm, "rgba": rgba, "rgb8": rgb8, "agg": agg}


def render_cube(cam, cube, minBox, cubeDim, cubeInc, iso, light=(0.0, 512.0, 0.0)):
    n = cam.c.W * cam.c.H
    rgba = np.empty((n, 4), np.float32)
    oob = C.c_int64()
    c = np.ascontiguousarray(cube, np.float32)
    lib().orc_render_cube(C.byref(cam.c), c.ctypes.data, _I3(*minBox), _I3(*cubeDim), _I3(*cubeInc), iso,
                          orc_f3(*light), rgba.ctypes.data, C.byref(oob))
    return rgba, oob.value


def read_voxels(volume, s, e):
    vol = np.ascontiguousarray(volume, np.float32)
    out = np.empty([abs(e[i] - s[i]) for i in range(3)], np.float32)
    lib().orc_read_voxels(vol.ctypes.data, _I3(*vol.shape), _I3(*s), _I3(*e), out.ctypes.data)
    return out


def build_octree(volume, iso, path):
    vol = np.ascontiguousarray(volume)
    vtype = 1 if vol.dtype == np.uint8 else 0
    r = lib().orc_build_octree(vol.ctypes.data, vtype, _I3(*vol.shape), float(iso), path.encode())
    if r != 0:
        raise IOError("oracle: cannot write %s" % path)


def children_mask(level_words, father):
    e = np.ascontiguousarray(level_words, np.uint64)
    return lib().orc_children_mask(e.ctypes.data if e.size else None, int(e.size), int(father))


def coordinate_to_index(x, y, z, level, nLevels):
    return lib().orc_coordinate_to_index(x, y, z, level, nLevels)


def min_box(index, level, nLevels):
    out = _I3()
    lib().orc_min_box(index, level, nLevels, out)
    return tuple(out)


class LRU:
    """lruCache state machine (src/lruCache.cu)."""

    def __init__(self, numElements, numElementsCPU, levelOctree, levelCube):
        self._h = lib().orc_lru_create(numElements, numElementsCPU, levelOctree, levelCube)
        if not self._h:
            raise ValueError("LinkedList needs at least 2 elements per tier")

    def update(self, ids, states):
        ids = np.ascontiguousarray(ids, np.uint64)
        st = np.ascontiguousarray(states, np.uint8).copy()
        n = ids.size
        slot = np.full(n, -1, np.int32)
        cube = np.zeros(n, np.uint64)
        loads = np.zeros(n, np.uint64)
        k = lib().orc_lru_update(self._h, n, ids.ctypes.data, st.ctypes.data, slot.ctypes.data, cube.ctypes.data,
                                 loads.ctypes.data)
        return st, slot, cube, loads[:k]

    def stats(self):
        out = (C.c_int64 * 5)()
        lib().orc_lru_stats(self._h, out)
        return tuple(out)

    def __del__(self):
        try:
            lib().orc_lru_free(self._h)
        except Exception:
            pass
