/*
 * vt_oracle.h -- CPU oracle for the visualTur isosurface ray-casting path.
 *
 * TEST INFRASTRUCTURE ONLY.  This is a literal host restatement of the
 * reference's algorithm (carlosduelo/visualTur) used as the checker for the
 * CUDA product in visualtur_b200/.  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline / reference legs may load it.  The product never
 * links, calls or falls back to it.
 *
 * Every function cites the reference file:line it restates.  Arithmetic is
 * single-precision IEEE with no contraction (built with -ffp-contract=off);
 * the reference's host-side `rsqrtf` is `1/sqrtf` (inc/cutil_math.h), which
 * is the definition used here for `normalize`.
 *
 * Pinning: the hyperslab reader is pinned by the known-answer checks of
 * src/testFileManager.cu:8-100 (mirrored in tests/test_oracle_filemanager.py);
 * the renderer is pinned against outputs of the reference's own device code
 * built from its sources (oracle/ref_build.sh -> oracle/_ref/) and stored as
 * fixtures in tests/golden/.
 */
#ifndef VT_ORACLE_H
#define VT_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct { float x, y, z; } orc_f3;

/* Camera + Screen state (inc/Camera.hpp:12-64, inc/Screen.hpp). */
typedef struct {
    int H, W, numRayPixel;
    float distance, fov_h, fov_w;
    float h, w;                       /* screen extent, src/Screen.cpp:18-19 */
    orc_f3 look, up, right, position;
    float rotX, rotY, rotZ;
} orc_camera;

void orc_camera_init(orc_camera* c, int nRP, int H, int W, float d, float fov_h, float fov_w);
void orc_camera_move(orc_camera* c, orc_f3 dir);
void orc_camera_rotate_x(orc_camera* c, float angle);
void orc_camera_rotate_y(orc_camera* c, float angle);
void orc_camera_rotate_z(orc_camera* c, float angle);
void orc_camera_move_forward(orc_camera* c, float dist);
void orc_camera_move_upward(orc_camera* c, float dist);
void orc_camera_strafe_right(orc_camera* c, float dist);
/* visualTur::changeScreen order (src/visualTur.cu:83-90). */
void orc_camera_change_screen(orc_camera* c, int W, int H, float fovW, float fovH, float d);
/* cuda_updateRays (src/Camera.cu:59-72): W*H directions, pixel id i*W+j. */
void orc_camera_rays(const orc_camera* c, orc_f3* out);

/* Morton utilities (inc/mortonCodeUtil.hpp). */
uint64_t orc_coordinate_to_index(int x, int y, int z, int level, int nLevels);
int      orc_index_level(uint64_t index);
void     orc_min_box(uint64_t index, int level, int nLevels, int out[3]);

/* Octree file (src/Octree.cu:769-813, src/CreateOctree.cu:342-371). */
typedef struct orc_octree orc_octree;
int  orc_octree_load(const char* path, orc_octree** out);      /* 0 ok, <0 error */
void orc_octree_free(orc_octree* o);
void orc_octree_info(const orc_octree* o, float* iso, int* dimension, int realDim[3], int* nLevels);
int  orc_octree_level_size(const orc_octree* o, int level);
const uint64_t* orc_octree_level(const orc_octree* o, int level);

/* Device-variant child membership (src/Octree.cu:375-532 with :15-20,
 * :78-99, :134-142): returns an 8-bit mask of children of `father` that the
 * reference's range search accepts in the level array e[0..size). */
int orc_children_mask(const uint64_t* e, int size, uint64_t father);

/* Voxel volume: x slowest, z fastest, index z + y*dy + x*dy*dz. */
enum { ORC_F32 = 0, ORC_U8 = 1 };

typedef struct {
    int levelO;          /* octreeLevel: candidate node level */
    int levelC;          /* levelCubes: brick level */
    int cubeInc;         /* apron */
    float iso;
    orc_f3 light;        /* visualTur: (0,512,0), src/visualTur.cu:30 */
    int nthreads;        /* 0 = OpenMP default */
    int ray_begin, ray_end, ray_stride;   /* subset of ray ids; end<=0 -> all */
    const orc_f3* dirs;  /* optional per-ray directions (NULL: cuda_updateRays) */
    int refine;          /* 0: reference refinement; k: k bisection steps first */
} orc_render_params;

typedef struct {
    /* per ray (indexed by ray id); any may be NULL */
    uint64_t* node_id;   /* hit candidate Morton code at levelO, 0 if none */
    uint64_t* brick_id;  /* brick code at levelC, 0 if none */
    float*    t;         /* dot(Xhit - origin, dir) for hits, -1 otherwise */
    float*    normal;    /* 3 floats per ray */
    float*    rgba;      /* 4 floats per ray */
    uint8_t*  rgb8;      /* 3 bytes per ray */
    /* aggregates */
    int64_t rays, hits, samples, normal_samples, candidates, expansions;
    int64_t max_stack, stack_overflow_rays, oob_taps;
} orc_render_out;

/* Full-frame render with reference semantics: the per-ray result of the
 * iterate-until-PAINTED loop of visualTur::updateVisibleCubes
 * (src/visualTur.cu:167-228) with enough cache and apron: DFS candidates
 * (src/Octree.cu:620-739) marched in order by cuda_rayCaster
 * (src/rayCaster.cu:139-265) sampling bricks read zero-padded
 * (src/FileManager.cu:86-167, src/lruCache.cu:223-226). */
int orc_render_frame(const orc_octree* o, const void* vol, int vtype, const int realDim[3],
                     const orc_camera* cam, const orc_render_params* p, orc_render_out* out);

/* cuda_rayCasterCube (src/rayCaster.cu:267-357): one resident brick. */
void orc_render_cube(const orc_camera* cam, const float* cube, const int minBox[3],
                     const int cubeDim[3], const int cubeInc[3], float iso, orc_f3 light,
                     float* rgba, int64_t* oob_taps);

/* FileManager::readHDF5_Voxel_Array (src/FileManager.cu:86-167). */
void orc_read_voxels(const float* vol, const int dims[3], const int s[3], const int e[3], float* out);

/* OctreeM builder (src/CreateOctree.cu:300-573); writes the octree file. */
int orc_build_octree(const void* vol, int vtype, const int realDim[3], float iso, const char* path);

/* lruCache state machine (src/lruCache.cu:7-313).  Host-only emulation:
 * slot numbers instead of pointers, no data movement. */
typedef struct orc_lru orc_lru;
orc_lru* orc_lru_create(int numElements, int numElementsCPU, int levelOctree, int levelCube);
void     orc_lru_free(orc_lru* c);
/* updateCache over num entries: state in/out (0/1/2/4/8), slot out (GPU
 * slot or -1), cubeID out; cpu_loads out: brick ids read from the volume
 * in order (capacity num), returns their count. */
int      orc_lru_update(orc_lru* c, int num, const uint64_t* id, uint8_t* state, int* slot,
                        uint64_t* cubeID, uint64_t* cpu_loads);
void     orc_lru_stats(const orc_lru* c, int64_t out[5]);  /* access hitsCPU missCPU hitsGPU missGPU */

#ifdef __cplusplus
}
#endif
#endif
