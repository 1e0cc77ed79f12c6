"""visualtur_b200 -- B200 (sm_100a) isosurface ray caster with the capabilities
of carlosduelo/visualTur.

The product is libvt.so (CUDA kernels + C ABI, include/vt.h) built from
csrc/ by build.py.  This module is a ctypes mirror of that ABI plus thin
classes keeping the reference's call surface (visualTur, FileManager,
Octree, Camera, rayCaster; inc/*.hpp of the reference).  There is no Python
or CPU fallback: every call goes to libvt.so, and loading fails loudly when
the library is missing.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libvt.so")

VT_OK, VT_ERR_INVALID, VT_ERR_CUDA, VT_ERR_IO, VT_ERR_FORMAT = 0, 1, 2, 3, 4
VT_ERR_NOMEM, VT_ERR_TIMEOUT, VT_ERR_STACK, VT_ERR_UNSUPPORTED, VT_ERR_STATE = 5, 6, 7, 8, 9
VT_F32, VT_U8 = 0, 1
VT_GEN_SPHERE, VT_GEN_BLOBS, VT_GEN_FRACTAL_U8 = 0, 1, 2
CAM_MOVE, CAM_ROTX, CAM_ROTY, CAM_ROTZ, CAM_FORWARD, CAM_UPWARD, CAM_STRAFE = range(7)


READ_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_void_p)


class VtError(RuntimeError):
    def __init__(self, status, msg):
        super().__init__("vt status %d: %s" % (status, msg))
        self.status = status


class vt_camera(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("distance", C.c_float), ("h", C.c_float), ("w", C.c_float),
                ("look", C.c_float * 3), ("up", C.c_float * 3), ("right", C.c_float * 3),
                ("position", C.c_float * 3)]


class vt_params(C.Structure):
    _fields_ = [("W", C.c_int), ("H", C.c_int), ("distance", C.c_float), ("fov_H", C.c_float),
                ("fov_W", C.c_float), ("numRayPx", C.c_int), ("maxElementsCache", C.c_int),
                ("maxElementsCache_CPU", C.c_int), ("dimCubeCache", C.c_int * 3), ("cubeInc", C.c_int),
                ("levelCubes", C.c_int), ("hdf5File", C.c_char_p), ("dataset_name", C.c_char_p),
                ("octreeFile", C.c_char_p), ("octreeLevel", C.c_int)]


class vt_options(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("resident", "tile_w", "tile_h", "unroll", "lookahead", "max_passes",
                                         "host_threads", "record_trace", "trace_level", "record_hits",
                                         "persistent", "blocks_per_sm", "pops", "preload", "use_graph", "refine",
                                         "skip", "max_suspended", "max_requests", "pool_per_ray", "spec_async",
                                         "wavefront", "shared_aprons", "demand_batch")]


class vt_stats(C.Structure):
    _fields_ = [(n, C.c_int64) for n in (
        "frames", "rays", "hits", "samples", "normal_samples", "candidates", "expansions", "passes",
        "bricks_requested", "bricks_loaded_host", "bricks_loaded_disk", "bricks_prefetched",
        "device_hits", "device_misses", "host_hits", "host_misses", "max_stack", "launches",
        "bricks_hinted", "bricks_staged", "bricks_speculative")] + \
        [(n, C.c_double) for n in ("ms_last_frame", "ms_stall_last_frame", "bytes_h2d_last_frame",
                                   "ms_trace_last_frame", "ms_prefetch_last_frame", "ms_host_read_total",
                                   "ms_fill_wait_total", "ms_wait_last_frame")] + \
        [("requests_deferred", C.c_int64), ("bricks_spec_loaded", C.c_int64)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class vt_h5_info(C.Structure):
    _fields_ = [("rank", C.c_int), ("dims", C.c_int64 * 32), ("type_class", C.c_int), ("type_size", C.c_int),
                ("is_signed", C.c_int), ("big_endian", C.c_int), ("offset", C.c_uint64), ("bytes", C.c_uint64)]


class vt_tuning(C.Structure):
    _fields_ = [(n, C.c_int) for n in ("tile_w", "tile_h", "unroll", "persistent", "pops", "blocks_per_sm",
                                         "lookahead", "use_graph", "skip", "spec_async", "wavefront",
                                         "shared_aprons", "demand_batch")]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class vt_view(C.Structure):
    _fields_ = [("cam", vt_camera), ("dev_rgba", C.c_void_p), ("dev_rgb8", C.c_void_p)]


_P = C.c_void_p
_I64_3 = C.c_int64 * 3
_PROTOS = {
    "vt_status_string": (C.c_char_p, [C.c_int]),
    "vt_last_error": (C.c_char_p, []),
    "vt_api_version": (C.c_int, []),
    "vt_volume_open": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(_P)]),
    "vt_volume_wrap": (C.c_int, [_P, C.c_int, _I64_3, C.POINTER(_P)]),
    "vt_volume_from_reader": (C.c_int, [_P, _P, C.c_int, _I64_3, C.POINTER(_P)]),
    "vt_volume_close": (None, [_P]),
    "vt_volume_info": (C.c_int, [_P, _I64_3, C.POINTER(C.c_int)]),
    "vt_volume_read": (C.c_int, [_P, C.c_int * 3, C.c_int * 3, _P]),
    "vt_volume_read_all": (C.c_int, [_P, _P]),
    "vt_volume_write": (C.c_int, [C.c_char_p, C.c_char_p, C.c_int, _P, C.c_int, _I64_3]),
    "vt_h5_describe": (C.c_int, [C.c_char_p, C.c_char_p, C.POINTER(vt_h5_info)]),
    "vt_generate_volume": (C.c_int, [C.c_int, C.c_uint64, _I64_3, _P, C.c_int, _P]),
    "vt_generate_volume_device": (C.c_int, [C.c_int, C.c_uint64, _I64_3, _P, C.c_int, _P, _P]),
    "vt_octree_load": (C.c_int, [C.c_char_p, C.POINTER(_P)]),
    "vt_octree_free": (None, [_P]),
    "vt_octree_info": (C.c_int, [_P, C.POINTER(C.c_float), C.POINTER(C.c_int), C.c_int * 3, C.POINTER(C.c_int)]),
    "vt_octree_level": (C.c_int, [_P, C.c_int, C.POINTER(C.c_int64), _P]),
    "vt_octree_build": (C.c_int, [_P, C.c_float, C.c_char_p, _P]),
    "vt_octree_build_device": (C.c_int, [_P, C.c_int, _I64_3, C.c_float, C.c_char_p, _P]),
    "vt_camera_init": (C.c_int, [C.POINTER(vt_camera), C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]),
    "vt_camera_op": (C.c_int, [C.POINTER(vt_camera), C.c_int, C.c_float, C.c_float, C.c_float]),
    "vt_camera_rays": (C.c_int, [C.POINTER(vt_camera), _P, _P]),
    "vt_render_cube": (C.c_int, [C.POINTER(vt_camera), _P, C.c_int * 3, C.c_int * 3, C.c_int * 3, C.c_float,
                                 C.c_float * 3, _P, _P]),
    "vt_default_options": (None, [C.POINTER(vt_options)]),
    "vt_create": (C.c_int, [C.POINTER(vt_params), C.POINTER(vt_options), C.POINTER(_P)]),
    "vt_create_from": (C.c_int, [C.POINTER(vt_params), C.POINTER(vt_options), _P, _P, C.POINTER(_P)]),
    "vt_destroy": (None, [_P]),
    "vt_camera_update": (C.c_int, [_P, C.c_int, C.c_float, C.c_float, C.c_float]),
    "vt_set_camera": (C.c_int, [_P, C.POINTER(vt_camera)]),
    "vt_get_camera": (C.c_int, [_P, C.POINTER(vt_camera)]),
    "vt_change_screen": (C.c_int, [_P, C.c_int, C.c_int, C.c_float, C.c_float, C.c_float]),
    "vt_change_num_rays": (C.c_int, [_P, C.c_int]),
    "vt_change_cache": (C.c_int, [_P, C.c_int, C.c_int * 3, C.c_int]),
    "vt_render": (C.c_int, [_P, _P, _P, _P]),
    "vt_render_host": (C.c_int, [_P, _P, _P]),
    "vt_render_batch": (C.c_int, [_P, C.POINTER(vt_view), C.c_int, _P]),
    "vt_debug_hits": (C.c_int, [_P, _P, _P, _P, _P]),
    "vt_get_trace": (C.c_int, [_P, _P, C.c_int64]),
    "vt_prefetch": (C.c_int, [_P, _P, C.c_int64, C.POINTER(C.c_int64), _P]),
    "vt_brick_list": (C.c_int, [_P, _P, C.POINTER(C.c_int64)]),
    "vt_debug_slot": (C.c_int, [_P, C.c_uint64, _P, C.POINTER(C.c_int)]),
    "vt_prefetch_hint": (C.c_int, [_P, _P, C.c_int64]),
    "vt_set_tuning": (C.c_int, [_P, C.POINTER(vt_tuning)]),
    "vt_drop_cache": (C.c_int, [_P]),
    "vt_get_tuning": (C.c_int, [_P, C.POINTER(vt_tuning)]),
    "vt_get_stats": (C.c_int, [_P, C.POINTER(vt_stats)]),
    "vt_reset_stats": (C.c_int, [_P]),
    "vt_mlp_create": (C.c_int, [C.c_int, C.c_int, C.c_int, C.c_int, C.c_uint64, C.POINTER(_P)]),
    "vt_mlp_free": (None, [_P]),
    "vt_mlp_forward": (C.c_int, [_P, _P, C.c_int, _P, _P]),
    "vt_mlp_train_step": (C.c_int, [_P, _P, _P, C.c_int, C.c_float, C.POINTER(C.c_float), _P]),
    "vt_mlp_gradients": (C.c_int, [_P, _P, _P, C.c_int, _P, C.POINTER(C.c_float)]),
    "vt_mlp_get_weights": (C.c_int, [_P, _P, C.POINTER(C.c_int64)]),
    "vt_mlp_set_weights": (C.c_int, [_P, _P, C.c_int64]),
    "vt_mlp_forward_noalloc": (C.c_int, [_P, _P, C.c_int, _P, _P]),
    "vt_mlp_info": (C.c_int, [_P, C.c_int * 4]),
    "vt_mlp_use_tensor_cores": (C.c_int, [_P, C.c_int]),
    "vt_prefetch_predict": (C.c_int, [_P, _P, C.POINTER(vt_camera), C.c_int, C.c_float, C.c_float, C.c_float, _P]),
}

_lib = None


def lib():
    """Loads libvt.so (once).  Raises if it has not been built."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError("libvt.so is not built (%s); run `python -m visualtur_b200.build`" % LIB_PATH)
        L = C.CDLL(LIB_PATH)
        for name, (res, args) in _PROTOS.items():
            f = getattr(L, name)
            f.restype = res
            f.argtypes = args
        _lib = L
    return _lib


def check(status):
    if status != VT_OK:
        raise VtError(status, lib().vt_last_error().decode(errors="replace"))


def _ptr(a):
    """Device/host pointer of a numpy array or torch tensor (or int/None)."""
    if a is None:
        return None
    if isinstance(a, int):
        return a
    if hasattr(a, "data_ptr"):
        return a.data_ptr()
    return a.ctypes.data


def _i3(v):
    return (C.c_int * 3)(*[int(x) for x in v])


def _d3(v):
    return _I64_3(*[int(x) for x in v])


# --------------------------------------------------------------------------- volumes
class FileManager:
    """Volume I/O with the reference's FileManager surface (inc/FileManager.hpp)."""

    def __init__(self, file_name=None, dataset_name="value", _handle=None, _keep=None):
        h = C.c_void_p()
        if _handle is not None:
            h = _handle
        else:
            check(lib().vt_volume_open(file_name.encode(), dataset_name.encode(), C.byref(h)))
        self._h = h
        self._keep = _keep
        d = _I64_3()
        vt = C.c_int()
        check(lib().vt_volume_info(self._h, d, C.byref(vt)))
        self.dims = tuple(int(x) for x in d)
        self.vtype = vt.value

    @classmethod
    def wrap(cls, array):
        """Wraps a host numpy volume (float32 or uint8, C order [x][y][z])."""
        a = np.ascontiguousarray(array)
        vt = VT_U8 if a.dtype == np.uint8 else VT_F32
        if vt == VT_F32 and a.dtype != np.float32:
            raise TypeError("volume must be float32 or uint8")
        h = C.c_void_p()
        check(lib().vt_volume_wrap(a.ctypes.data, vt, _d3(a.shape), C.byref(h)))
        return cls(_handle=h, _keep=a)

    @classmethod
    def from_reader(cls, read, dims, vtype=VT_F32):
        """A volume read through `read(s, e) -> array or None`: the voxels
        [s, e) as readHDF5_Voxel_Array returns them (zeros outside the
        volume), or None when the read fails (the render call then raises
        VtError with VT_ERR_IO).  Called from libvt's host threads."""
        dt = np.uint8 if vtype == VT_U8 else np.float32

        def cb(user, s, e, out):
            try:
                box = read(tuple(s[i] for i in range(3)), tuple(e[i] for i in range(3)))
                if box is None:
                    return 1
                b = np.ascontiguousarray(box, dt)
                C.memmove(out, b.ctypes.data, b.nbytes)
                return 0
            except Exception:
                return 1
        fn = READ_FN(cb)
        h = C.c_void_p()
        check(lib().vt_volume_from_reader(C.cast(fn, C.c_void_p), None, vtype, _d3(dims), C.byref(h)))
        return cls(_handle=h, _keep=fn)

    def readHDF5_Voxel_Array(self, s, e):
        out = np.empty([abs(int(e[i]) - int(s[i])) for i in range(3)], np.float32)
        check(lib().vt_volume_read(self._h, _i3(s), _i3(e), out.ctypes.data))
        return out

    def readHDF5(self):
        out = np.empty(self.dims, np.uint8 if self.vtype == VT_U8 else np.float32)
        check(lib().vt_volume_read_all(self._h, out.ctypes.data))
        return out

    @staticmethod
    def CreateFile(volume, newname, dataset_name="value", fmt=1):
        """Writes the volume as an HDF5 file with one contiguous dataset
        (fmt 1, as FileManager::CreateFile) or as a raw VTVOL001 file (fmt 0)."""
        a = np.ascontiguousarray(volume)
        vt = VT_U8 if a.dtype == np.uint8 else VT_F32
        check(lib().vt_volume_write(newname.encode(), dataset_name.encode(), fmt, a.ctypes.data, vt, _d3(a.shape)))

    @staticmethod
    def h5_describe(path, dataset="value"):
        """The HDF5 dataset as libvt's reader sees it: rank, dims, element
        class ("int"/"float"), size, signedness, byte order, file offset."""
        i = vt_h5_info()
        check(lib().vt_h5_describe(path.encode(), dataset.encode(), C.byref(i)))
        return {"rank": i.rank, "dims": tuple(int(i.dims[k]) for k in range(i.rank)),
                "class": "float" if i.type_class == 1 else "int", "size": i.type_size,
                "signed": bool(i.is_signed), "big_endian": bool(i.big_endian),
                "offset": int(i.offset), "bytes": int(i.bytes)}

    def close(self):
        if self._h:
            lib().vt_volume_close(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def generate_volume(kind, seed, dims, params=(), device_ptr=None, stream=None):
    """Seeded synthetic volume; on the host (numpy) unless device_ptr given."""
    prm = np.asarray(params, np.float32)
    if device_ptr is not None:
        check(lib().vt_generate_volume_device(kind, seed, _d3(dims), prm.ctypes.data if prm.size else None,
                                              int(prm.size), device_ptr, stream))
        return None
    out = np.empty(tuple(int(d) for d in dims), np.uint8 if kind == VT_GEN_FRACTAL_U8 else np.float32)
    check(lib().vt_generate_volume(kind, seed, _d3(dims), prm.ctypes.data if prm.size else None, int(prm.size),
                                   out.ctypes.data))
    return out


# --------------------------------------------------------------------------- octree
class Octree:
    """Octree file (src/Octree.cu:769-813)."""

    def __init__(self, file_name):
        self._h = C.c_void_p()
        check(lib().vt_octree_load(file_name.encode(), C.byref(self._h)))
        iso, dim, nl = C.c_float(), C.c_int(), C.c_int()
        rd = (C.c_int * 3)()
        check(lib().vt_octree_info(self._h, C.byref(iso), C.byref(dim), rd, C.byref(nl)))
        self.isosurface, self.dimension, self.nLevels = iso.value, dim.value, nl.value
        self.realDim = tuple(rd)

    def getIsosurface(self):
        return self.isosurface

    def getnLevels(self):
        return self.nLevels

    def level(self, l):
        n = C.c_int64()
        check(lib().vt_octree_level(self._h, l, C.byref(n), None))
        out = np.empty(n.value, np.uint64)
        check(lib().vt_octree_level(self._h, l, C.byref(n), out.ctypes.data))
        return out

    def close(self):
        if self._h:
            lib().vt_octree_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def build_octree(fm, iso, path, stream=None):
    """OctreeM + writeToFile on the GPU."""
    check(lib().vt_octree_build(fm._h, float(iso), path.encode(), stream))


def build_octree_device(dev_ptr, vtype, dims, iso, path, stream=None):
    """Same for a volume already on the device."""
    check(lib().vt_octree_build_device(dev_ptr, vtype, _d3(dims), float(iso), path.encode(), stream))


# --------------------------------------------------------------------------- camera
class Camera:
    """Camera state with the reference's operations (src/Camera.cu)."""

    def __init__(self, H, W, distance, fov_H, fov_W, _cam=None):
        self.c = vt_camera()
        if _cam is not None:
            self.c = _cam
        else:
            check(lib().vt_camera_init(C.byref(self.c), H, W, distance, fov_H, fov_W))

    def _op(self, op, a=0.0, b=0.0, c=0.0):
        check(lib().vt_camera_op(C.byref(self.c), op, a, b, c))

    def Move(self, d):
        self._op(CAM_MOVE, *d)

    def RotateX(self, a):
        self._op(CAM_ROTX, a)

    def RotateY(self, a):
        self._op(CAM_ROTY, a)

    def RotateZ(self, a):
        self._op(CAM_ROTZ, a)

    def MoveForward(self, d):
        self._op(CAM_FORWARD, d)

    def MoveUpward(self, d):
        self._op(CAM_UPWARD, d)

    def StrafeRight(self, d):
        self._op(CAM_STRAFE, d)

    def rays_into(self, dev_dirs, stream=None):
        check(lib().vt_camera_rays(C.byref(self.c), _ptr(dev_dirs), stream))

    def state(self):
        c = self.c
        return {"look": tuple(c.look), "up": tuple(c.up), "right": tuple(c.right),
                "position": tuple(c.position), "h": c.h, "w": c.w}


class rayCaster:
    """rayCaster::renderCube (src/rayCaster.cu:385-394)."""

    def __init__(self, isosurface, lposition=(0.0, 512.0, 0.0)):
        self.iso = float(isosurface)
        self.light = (C.c_float * 3)(*lposition)

    def renderCube(self, camera, dev_cube, minBox, cubeDim, cubeInc, dev_buffer, stream=None):
        check(lib().vt_render_cube(C.byref(camera.c), _ptr(dev_cube), _i3(minBox), _i3(cubeDim), _i3(cubeInc),
                                   self.iso, self.light, _ptr(dev_buffer), stream))


def default_options(**kw):
    o = vt_options()
    lib().vt_default_options(C.byref(o))
    for k, v in kw.items():
        setattr(o, k, v)
    return o


def make_params(W, H, octreeFile, hdf5File, octreeLevel, levelCubes, dimCube, cubeInc=3, distance=50.0,
                fov_H=30.0, fov_W=30.0, maxElementsCache=4096, maxElementsCache_CPU=4096, dataset="value"):
    p = vt_params()
    p.W, p.H, p.distance, p.fov_H, p.fov_W, p.numRayPx = W, H, distance, fov_H, fov_W, 1
    p.maxElementsCache, p.maxElementsCache_CPU = maxElementsCache, maxElementsCache_CPU
    p.dimCubeCache = (C.c_int * 3)(dimCube, dimCube, dimCube)
    p.cubeInc, p.levelCubes, p.octreeLevel = cubeInc, levelCubes, octreeLevel
    p.hdf5File = hdf5File.encode() if hdf5File else None
    p.dataset_name = dataset.encode()
    p.octreeFile = octreeFile.encode() if octreeFile else None
    return p


class visualTur:
    """Renderer with the reference's visualTur surface (inc/visualTur.hpp)."""

    def __init__(self, params, options=None, volume=None, octree=None):
        self._h = C.c_void_p()
        self._keep = (params, volume, octree)
        opt = options if options is not None else default_options()
        if volume is not None:
            check(lib().vt_create_from(C.byref(params), C.byref(opt), volume._h, octree._h, C.byref(self._h)))
        else:
            check(lib().vt_create(C.byref(params), C.byref(opt), C.byref(self._h)))
        self.W, self.H = params.W, params.H

    def _cam(self, op, a=0.0, b=0.0, c=0.0):
        check(lib().vt_camera_update(self._h, op, a, b, c))

    def camera_Move(self, d):
        self._cam(CAM_MOVE, *d)

    def camera_RotateX(self, a):
        self._cam(CAM_ROTX, a)

    def camera_RotateY(self, a):
        self._cam(CAM_ROTY, a)

    def camera_RotateZ(self, a):
        self._cam(CAM_ROTZ, a)

    def camera_MoveForward(self, d):
        self._cam(CAM_FORWARD, d)

    def camera_MoveUpward(self, d):
        self._cam(CAM_UPWARD, d)

    def camera_StrafeRight(self, d):
        self._cam(CAM_STRAFE, d)

    def get_camera(self):
        c = vt_camera()
        check(lib().vt_get_camera(self._h, C.byref(c)))
        return c

    def set_camera(self, c):
        check(lib().vt_set_camera(self._h, C.byref(c)))

    def changeScreen(self, W, H, fovW, fovH, distance):
        check(lib().vt_change_screen(self._h, W, H, fovW, fovH, distance))
        self.W, self.H = W, H

    def changeNumRays(self, n):
        check(lib().vt_change_num_rays(self._h, n))

    def changeCacheParameters(self, nE, cDim, cInc):
        check(lib().vt_change_cache(self._h, nE, _i3(cDim), cInc))

    def updateVisibleCubes(self, dev_rgba, dev_rgb8=None, stream=None):
        """Renders into caller device buffers (both None: the handle's own)."""
        check(lib().vt_render(self._h, _ptr(dev_rgba), _ptr(dev_rgb8), stream))

    def render_host(self, rgb8=True):
        rgba = np.empty((self.H * self.W, 4), np.float32)
        out8 = np.empty((self.H * self.W, 3), np.uint8) if rgb8 else None
        check(lib().vt_render_host(self._h, rgba.ctypes.data, out8.ctypes.data if rgb8 else None))
        return rgba, out8

    def render_batch(self, views, stream=None):
        arr = (vt_view * len(views))(*views)
        check(lib().vt_render_batch(self._h, arr, len(views), stream))

    def debug_hits(self):
        n = self.W * self.H
        node = np.empty(n, np.uint64)
        brick = np.empty(n, np.uint64)
        t = np.empty(n, np.float32)
        nrm = np.empty((n, 3), np.float32)
        check(lib().vt_debug_hits(self._h, node.ctypes.data, brick.ctypes.data, t.ctypes.data, nrm.ctypes.data))
        return node, brick, t, nrm

    def trace(self, level=4):
        nw = max(1, (8 ** level) // 32)
        out = np.empty(nw, np.uint32)
        check(lib().vt_get_trace(self._h, out.ctypes.data, nw))
        return out

    def prefetch(self, bricks, stream=None):
        b = np.ascontiguousarray(bricks, np.uint64)
        got = C.c_int64()
        check(lib().vt_prefetch(self._h, b.ctypes.data, int(b.size), C.byref(got), stream))
        return got.value

    def tuning(self):
        t = vt_tuning()
        check(lib().vt_get_tuning(self._h, C.byref(t)))
        return t.as_dict()

    def set_tuning(self, **kw):
        t = vt_tuning()
        check(lib().vt_get_tuning(self._h, C.byref(t)))
        for k, v in kw.items():
            setattr(t, k, int(v))
        check(lib().vt_set_tuning(self._h, C.byref(t)))

    def prefetch_hint(self, bricks):
        b = np.ascontiguousarray(bricks, np.uint64)
        check(lib().vt_prefetch_hint(self._h, b.ctypes.data if b.size else None, int(b.size)))

    def prefetch_predict(self, mlp, cams, vol_edge, fov, threshold, stream=None):
        """Learned prefetch on the device (vt_prefetch_predict): the network
        `mlp` predicts, from the poses `cams`, the bricks the coming frames
        march; absent ones are requested speculatively and load while the
        next render call's passes run.  Nothing is synchronised or copied
        back to Python."""
        arr = (vt_camera * len(cams))(*cams)
        check(lib().vt_prefetch_predict(self._h, mlp._h, arr, len(cams), float(vol_edge), float(fov), float(threshold),
                                        stream))

    def brick_list(self):
        n = C.c_int64(0)
        check(lib().vt_brick_list(self._h, None, C.byref(n)))
        out = np.empty(n.value, np.uint64)
        check(lib().vt_brick_list(self._h, out.ctypes.data, C.byref(n)))
        return out

    def debug_slot(self, code, D, dtype):
        """The device-cache slot of brick `code` as a D x D x D array of
        `dtype`, or None when the brick has no slot."""
        out = np.empty((D, D, D), dtype)
        res = C.c_int(0)
        check(lib().vt_debug_slot(self._h, int(code), out.ctypes.data, C.byref(res)))
        return out if res.value else None

    def stats(self):
        s = vt_stats()
        check(lib().vt_get_stats(self._h, C.byref(s)))
        return s.as_dict()

    def reset_stats(self):
        check(lib().vt_reset_stats(self._h))

    def drop_cache(self):
        check(lib().vt_drop_cache(self._h))

    def close(self):
        if self._h:
            lib().vt_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class MLP:
    """Prefetch network (vt_mlp_*): in -> h1 -> h2 -> out, BF16 weights, FP32
    accumulation, trained on the GPU by libvt's own kernels."""

    def __init__(self, dims=(12, 512, 512, 4096), seed=0):
        self.dims = tuple(int(d) for d in dims)
        self._h = C.c_void_p()
        check(lib().vt_mlp_create(*self.dims, seed, C.byref(self._h)))

    def use_tensor_cores(self, on=True):
        """GEMMs on the tensor cores (default) or on the SIMT FMA pipes."""
        check(lib().vt_mlp_use_tensor_cores(self._h, 1 if on else 0))
        self.tensor_cores = bool(on)

    tensor_cores = True

    def forward(self, dev_x, batch, dev_p, stream=None):
        check(lib().vt_mlp_forward(self._h, _ptr(dev_x), batch, _ptr(dev_p), stream))

    def forward_noalloc(self, dev_x, batch, dev_p, stream=None):
        """Same result as forward(); allocates nothing (fixed 1 MiB device
        scratch, batch * (h1 + h2) <= 262144; calls must not overlap)."""
        check(lib().vt_mlp_forward_noalloc(self._h, _ptr(dev_x), batch, _ptr(dev_p), stream))

    def train_step(self, dev_x, dev_y, batch, lr, stream=None, want_loss=True):
        loss = C.c_float()
        check(lib().vt_mlp_train_step(self._h, _ptr(dev_x), _ptr(dev_y), batch, lr,
                                      C.byref(loss) if want_loss else None, stream))
        return loss.value

    def gradients(self, dev_x, dev_y, batch):
        n = C.c_int64(0)
        check(lib().vt_mlp_get_weights(self._h, None, C.byref(n)))
        g = np.empty(n.value, np.float32)
        loss = C.c_float()
        check(lib().vt_mlp_gradients(self._h, _ptr(dev_x), _ptr(dev_y), batch, g.ctypes.data, C.byref(loss)))
        return self._split(g), loss.value

    def weights(self):
        n = C.c_int64(0)
        check(lib().vt_mlp_get_weights(self._h, None, C.byref(n)))
        w = np.empty(n.value, np.float32)
        check(lib().vt_mlp_get_weights(self._h, w.ctypes.data, C.byref(n)))
        return self._split(w)

    def set_weights(self, layers):
        flat = np.concatenate([np.ascontiguousarray(a, np.float32).ravel() for wb in layers for a in wb])
        check(lib().vt_mlp_set_weights(self._h, flat.ctypes.data, flat.size))

    def _split(self, flat):
        out, o, d = [], 0, self.dims
        for l in range(3):
            nw = d[l] * d[l + 1]
            out.append((flat[o:o + nw].reshape(d[l], d[l + 1]), flat[o + nw:o + nw + d[l + 1]]))
            o += nw + d[l + 1]
        return out

    def close(self):
        if self._h:
            lib().vt_mlp_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
