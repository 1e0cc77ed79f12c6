/*
 * visualtur.hpp -- header-only C++ facade over include/vt.h that keeps the
 * call surface of carlosduelo/visualTur's classes (inc/visualTur.hpp,
 * inc/FileManager.hpp, inc/Camera.hpp, inc/rayCaster.hpp, inc/Octree.hpp),
 * so code written against the reference compiles against libvt.so.
 *
 * Differences a caller sees: failures throw vt::Error (the reference prints
 * and calls exit(0) or throws std::exception); numRayPx must be 1 and
 * cubeInc >= 3 (see vt.h).  Define VT_REFERENCE_NAMES before including to
 * get the classes in the global namespace under the reference's names.
 */
#ifndef VISUALTUR_HPP
#define VISUALTUR_HPP

#include <vector_types.h>

#include <stdexcept>
#include <string>

#include "vt.h"

namespace vt {

struct Error : std::runtime_error {
    vt_status status;
    Error(vt_status s, const char* what) : std::runtime_error(what), status(s) {}
};
inline void check(vt_status s) {
    if (s != VT_OK) throw Error(s, vt_last_error());
}

/* visualTurParams_t (inc/visualTur.hpp:12-33) */
typedef struct {
    int W, H;
    float distance, fov_H, fov_W;
    int numRayPx;
    int maxElementsCache, maxElementsCache_CPU;
    int3 dimCubeCache;
    int cubeInc, levelCubes;
    char* hdf5File;
    char* dataset_name;
    char* octreeFile;
    int octreeLevel;
} visualTurParams_t;

/* FileManager (inc/FileManager.hpp:12-35) */
class FileManager {
public:
    unsigned long long dims[3];
    FileManager(const char* file_name, const char* dataset_name) {
        check(vt_volume_open(file_name, dataset_name, &v_));
        int64_t d[3];
        check(vt_volume_info(v_, d, nullptr));
        for (int i = 0; i < 3; i++) dims[i] = (unsigned long long)d[i];
    }
    ~FileManager() { vt_volume_close(v_); }
    FileManager(const FileManager&) = delete;
    FileManager& operator=(const FileManager&) = delete;
    int readHDF5(float* volume) { check(vt_volume_read_all(v_, volume)); return 0; }
    void readHDF5_Voxel_Array(int3 s, int3 e, float* data) {
        int a[3] = {s.x, s.y, s.z}, b[3] = {e.x, e.y, e.z};
        check(vt_volume_read(v_, a, b, data));
    }
    int CreateFile(float* volume, char* newname, char* dataset_name, int x, int y, int z) {
        int64_t d[3] = {x, y, z};
        check(vt_volume_write(newname, dataset_name, 1, volume, VT_F32, d));
        return 0;
    }
    vt_volume* handle() const { return v_; }

private:
    vt_volume* v_ = nullptr;
};

/* Camera (inc/Camera.hpp:12-64); directions are written on demand */
class Camera {
public:
    Camera(int nRP, int H, int W, float d, float fov_h, float fov_w) : fovH_(fov_h), fovW_(fov_w) {
        if (nRP != 1) throw Error(VT_ERR_UNSUPPORTED, "numRayPixel must be 1");
        check(vt_camera_init(&c_, H, W, d, fov_h, fov_w));
    }
    void Move(float3 d) { check(vt_camera_op(&c_, 0, d.x, d.y, d.z)); }
    void RotateX(float a) { check(vt_camera_op(&c_, 1, a, 0, 0)); }
    void RotateY(float a) { check(vt_camera_op(&c_, 2, a, 0, 0)); }
    void RotateZ(float a) { check(vt_camera_op(&c_, 3, a, 0, 0)); }
    void MoveForward(float d) { check(vt_camera_op(&c_, 4, d, 0, 0)); }
    void MoveUpward(float d) { check(vt_camera_op(&c_, 5, d, 0, 0)); }
    void StrafeRight(float d) { check(vt_camera_op(&c_, 6, d, 0, 0)); }
    int get_H() const { return c_.H; }
    int get_W() const { return c_.W; }
    float get_h() const { return c_.h; }
    float get_w() const { return c_.w; }
    float get_Distance() const { return c_.distance; }
    float get_fovH() const { return fovH_; }
    float get_fovW() const { return fovW_; }
    int get_numRayPixel() const { return 1; }
    int get_numRays() const { return c_.W * c_.H; }
    float3 get_look() const { return make(c_.look); }
    float3 get_up() const { return make(c_.up); }
    float3 get_right() const { return make(c_.right); }
    float3 get_position() const { return make(c_.position); }
    /* cuda_updateRays into a caller-owned device buffer of W*H float3 */
    void rayDirections(float3* dev, void* stream = nullptr) const { check(vt_camera_rays(&c_, (float*)dev, stream)); }
    const vt_camera& desc() const { return c_; }

private:
    static float3 make(const float* a) { float3 r; r.x = a[0]; r.y = a[1]; r.z = a[2]; return r; }
    vt_camera c_;
    float fovH_, fovW_;
};

/* rayCaster (inc/rayCaster.hpp:12-30): renderCube */
class rayCaster {
public:
    rayCaster(float isosurface, float3 lposition) : iso_(isosurface) {
        l_[0] = lposition.x; l_[1] = lposition.y; l_[2] = lposition.z;
    }
    void renderCube(Camera* camera, float* cube, int3 minBox, int3 cubeDim, int3 cubeInc, float* buffer,
                    void* stream = nullptr) {
        int a[3] = {minBox.x, minBox.y, minBox.z}, b[3] = {cubeDim.x, cubeDim.y, cubeDim.z};
        int c[3] = {cubeInc.x, cubeInc.y, cubeInc.z};
        check(vt_render_cube(&camera->desc(), cube, a, b, c, iso_, l_, buffer, stream));
    }

private:
    float iso_;
    float l_[3];
};

/* Octree file (inc/Octree.hpp:12-42) */
class Octree {
public:
    explicit Octree(const char* file_name) { check(vt_octree_load(file_name, &o_)); }
    ~Octree() { vt_octree_free(o_); }
    Octree(const Octree&) = delete;
    Octree& operator=(const Octree&) = delete;
    int getnLevels() const { int n; check(vt_octree_info(o_, nullptr, nullptr, nullptr, &n)); return n; }
    float getIsosurface() const { float i; check(vt_octree_info(o_, &i, nullptr, nullptr, nullptr)); return i; }

private:
    vt_octree* o_ = nullptr;
};

/* visualTur (inc/visualTur.hpp:35-80) */
class visualTur {
public:
    explicit visualTur(visualTurParams_t p, const vt_options* opt = nullptr) {
        vt_params q;
        q.W = p.W; q.H = p.H; q.distance = p.distance; q.fov_H = p.fov_H; q.fov_W = p.fov_W;
        q.numRayPx = p.numRayPx; q.maxElementsCache = p.maxElementsCache;
        q.maxElementsCache_CPU = p.maxElementsCache_CPU;
        q.dimCubeCache[0] = p.dimCubeCache.x; q.dimCubeCache[1] = p.dimCubeCache.y; q.dimCubeCache[2] = p.dimCubeCache.z;
        q.cubeInc = p.cubeInc; q.levelCubes = p.levelCubes;
        q.hdf5File = p.hdf5File; q.dataset_name = p.dataset_name; q.octreeFile = p.octreeFile;
        q.octreeLevel = p.octreeLevel;
        check(vt_create(&q, opt, &h_));
    }
    ~visualTur() { vt_destroy(h_); }
    visualTur(const visualTur&) = delete;
    visualTur& operator=(const visualTur&) = delete;
    void changeScreen(int W, int H, float fovW, float fovH, float d) { check(vt_change_screen(h_, W, H, fovW, fovH, d)); }
    void changeNumRays(int n) { check(vt_change_num_rays(h_, n)); }
    void changeCacheParameters(int nE, int3 cDim, int cInc) {
        int d[3] = {cDim.x, cDim.y, cDim.z};
        check(vt_change_cache(h_, nE, d, cInc));
    }
    void camera_Move(float3 d) { check(vt_camera_update(h_, 0, d.x, d.y, d.z)); }
    void camera_RotateX(float a) { check(vt_camera_update(h_, 1, a, 0, 0)); }
    void camera_RotateY(float a) { check(vt_camera_update(h_, 2, a, 0, 0)); }
    void camera_RotateZ(float a) { check(vt_camera_update(h_, 3, a, 0, 0)); }
    void camera_MoveForward(float d) { check(vt_camera_update(h_, 4, d, 0, 0)); }
    void camera_MoveUpward(float d) { check(vt_camera_update(h_, 5, d, 0, 0)); }
    void camera_StrafeRight(float d) { check(vt_camera_update(h_, 6, d, 0, 0)); }
    /* device buffer of W*H*4 floats, as in the reference */
    void updateVisibleCubes(float* pixelBuffer, void* stream = nullptr) { check(vt_render(h_, pixelBuffer, nullptr, stream)); }
    vt_handle* handle() const { return h_; }

private:
    vt_handle* h_ = nullptr;
};

}  // namespace vt

#ifdef VT_REFERENCE_NAMES
using vt::Camera;
using vt::FileManager;
using vt::Octree;
using vt::rayCaster;
using vt::visualTur;
using vt::visualTurParams_t;
#endif

#endif
