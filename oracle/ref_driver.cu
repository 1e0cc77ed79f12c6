/*
 * ref_driver.cu -- runs the reference's own classes, compiled from its
 * sources by oracle/ref_build.sh, on seeded inputs and dumps their outputs
 * as raw arrays.  TEST INFRASTRUCTURE: its only use is to generate the
 * golden vectors in tests/golden/ that pin the CPU oracle.
 *
 *   vtref render VOL OCT W H fovH fovW dist levelC levelO inc nGPU nCPU OUT op...
 *       visualTur (inc/visualTur.hpp) + camera ops + updateVisibleCubes.
 *       ops: mv:x,y,z  rx:a  ry:a  rz:a  mf:d  mu:d  sr:d
 *       writes OUT.rgba (f32 x4), OUT.ids (u64), OUT.cube (u64),
 *       OUT.state (u8), OUT.dirs (f32 x3), OUT.cam (f32 x16), OUT.log
 *   vtref cube VOL W H dist fovH fovW px py pz bx by bz dim inc iso OUT
 *       testRayCaster-style rayCaster::renderCube (src/testRayCaster.cu).
 *       writes OUT.rgba, OUT.dirs
 *   vtref lru VOL nGPU nCPU levelO levelC nLevels inc SEQ OUT
 *       lruCache::updateCache over rounds read from SEQ (i32 rounds,
 *       i32 n, then per round n x (u64 id, u8 state)); writes OUT (per
 *       entry u8 state, i32 slot, u64 cubeID) and OUT.stats (5 x i64).
 *
 * A watchdog ends the process if a run exceeds its time limit.
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#include <chrono>
#include <string>
#include <thread>
#include <vector>

#include <cuda_runtime.h>

#define private public
#include "visualTur.hpp"
#undef private

static void die(const char* m) { fprintf(stdout, "vtref error: %s\n", m); fflush(stdout); _exit(2); }

static void dump(const std::string& path, const void* p, size_t n) {
    FILE* f = fopen(path.c_str(), "wb");
    if (!f || fwrite(p, 1, n, f) != n) die("write");
    fclose(f);
}

static void watchdog(int seconds) {
    std::thread([seconds]() {
        std::this_thread::sleep_for(std::chrono::seconds(seconds));
        fprintf(stdout, "vtref watchdog: time limit reached\n");
        fflush(stdout);
        _exit(3);
    }).detach();
}

static void apply_op(visualTur* vt, const char* op) {
    float a, b, c;
    if (sscanf(op, "mv:%f,%f,%f", &a, &b, &c) == 3) vt->camera_Move(make_float3(a, b, c));
    else if (sscanf(op, "rx:%f", &a) == 1) vt->camera_RotateX(a);
    else if (sscanf(op, "ry:%f", &a) == 1) vt->camera_RotateY(a);
    else if (sscanf(op, "rz:%f", &a) == 1) vt->camera_RotateZ(a);
    else if (sscanf(op, "mf:%f", &a) == 1) vt->camera_MoveForward(a);
    else if (sscanf(op, "mu:%f", &a) == 1) vt->camera_MoveUpward(a);
    else if (sscanf(op, "sr:%f", &a) == 1) vt->camera_StrafeRight(a);
    else die("bad op");
}

static int run_render(int argc, char** argv) {
    if (argc < 15) die("render: args");
    char* vol = argv[2];
    char* oct = argv[3];
    int W = atoi(argv[4]), H = atoi(argv[5]);
    float fovH = atof(argv[6]), fovW = atof(argv[7]), dist = atof(argv[8]);
    int levelC = atoi(argv[9]), levelO = atoi(argv[10]), inc = atoi(argv[11]);
    int nGPU = atoi(argv[12]), nCPU = atoi(argv[13]);
    std::string out = argv[14];

    FILE* f = fopen(oct, "rb");
    if (!f) die("octree open");
    int hdr[7];
    if (fread(hdr, 4, 7, f) != 7) die("octree header");
    fclose(f);
    int nLevels = hdr[6];
    int cd = 1 << (nLevels - levelC);

    visualTurParams_t p;
    p.W = W; p.H = H; p.fov_H = fovH; p.fov_W = fovW; p.distance = dist; p.numRayPx = 1;
    p.maxElementsCache = nGPU; p.maxElementsCache_CPU = nCPU;
    p.dimCubeCache = make_int3(cd, cd, cd); p.cubeInc = inc; p.levelCubes = levelC;
    p.hdf5File = vol; p.dataset_name = (char*)"value"; p.octreeFile = oct; p.octreeLevel = levelO;

    visualTur* vt = new visualTur(p);
    for (int i = 15; i < argc; i++) apply_op(vt, argv[i]);

    float* screenG = 0;
    size_t n = (size_t)W * H;
    if (cudaMalloc((void**)&screenG, n * 4 * sizeof(float)) != cudaSuccess) die("malloc screen");
    cudaMemset(screenG, 0, n * 4 * sizeof(float));
    vt->updateVisibleCubes(screenG);
    if (cudaDeviceSynchronize() != cudaSuccess) die("render sync");

    std::vector<float> rgba(n * 4), dirs(n * 3);
    cudaMemcpy(rgba.data(), screenG, n * 16, cudaMemcpyDeviceToHost);
    cudaMemcpy(dirs.data(), vt->camera->get_rayDirections(), n * 12, cudaMemcpyDeviceToHost);
    std::vector<unsigned long long> ids(n), cube(n);
    std::vector<unsigned char> st(n);
    for (size_t i = 0; i < n; i++) {
        ids[i] = vt->visibleCubesCPU[i].id;
        cube[i] = vt->visibleCubesCPU[i].cubeID;
        st[i] = vt->visibleCubesCPU[i].state;
    }
    float cam[16];
    float3 v[4] = {vt->camera->get_look(), vt->camera->get_up(), vt->camera->get_right(),
                   vt->camera->get_position()};
    for (int i = 0; i < 4; i++) { cam[3 * i] = v[i].x; cam[3 * i + 1] = v[i].y; cam[3 * i + 2] = v[i].z; }
    cam[12] = vt->camera->get_h(); cam[13] = vt->camera->get_w();
    cam[14] = (float)nLevels; cam[15] = vt->octree->getIsosurface();
    dump(out + ".rgba", rgba.data(), n * 16);
    dump(out + ".dirs", dirs.data(), n * 12);
    dump(out + ".ids", ids.data(), n * 8);
    dump(out + ".cube", cube.data(), n * 8);
    dump(out + ".state", st.data(), n);
    dump(out + ".cam", cam, sizeof(cam));
    cudaFree(screenG);
    delete vt;
    return 0;
}

static int run_cube(int argc, char** argv) {
    if (argc < 18) die("cube: args");
    char* vol = argv[2];
    int W = atoi(argv[3]), H = atoi(argv[4]);
    float dist = atof(argv[5]), fovH = atof(argv[6]), fovW = atof(argv[7]);
    float px = atof(argv[8]), py = atof(argv[9]), pz = atof(argv[10]);
    int bx = atoi(argv[11]), by = atoi(argv[12]), bz = atoi(argv[13]);
    int dim = atoi(argv[14]), inc = atoi(argv[15]);
    float iso = atof(argv[16]);
    std::string out = argv[17];

    Camera* camera = new Camera(1, H, W, dist, fovH, fovW);
    camera->Move(make_float3(px, py, pz));
    int3 coord = make_int3(bx, by, bz);
    int3 cubeDim = make_int3(dim, dim, dim);
    int3 cubeInc = make_int3(inc, inc, inc);
    int3 real = cubeDim + 2 * cubeInc;
    size_t nv = (size_t)real.x * real.y * real.z;
    std::vector<float> cpu(nv);
    float* gpu = 0;
    if (cudaMalloc((void**)&gpu, nv * 4) != cudaSuccess) die("malloc cube");
    int3 minBox = coord - cubeInc;
    int3 maxBox = minBox + real;
    FileManager* fm = new FileManager(vol, "value");
    fm->readHDF5_Voxel_Array(minBox, maxBox, cpu.data());
    cudaMemcpy(gpu, cpu.data(), nv * 4, cudaMemcpyHostToDevice);
    size_t n = (size_t)W * H;
    float* screen = 0;
    if (cudaMalloc((void**)&screen, n * 16) != cudaSuccess) die("malloc screen");
    rayCaster* rc = new rayCaster(iso, make_float3(0.0f, 512.0f, 0.0f));
    rc->renderCube(camera, gpu, make_int3(0, 0, 0), cubeDim, cubeInc, screen);
    if (cudaDeviceSynchronize() != cudaSuccess) die("cube sync");
    std::vector<float> rgba(n * 4), dirs(n * 3);
    cudaMemcpy(rgba.data(), screen, n * 16, cudaMemcpyDeviceToHost);
    cudaMemcpy(dirs.data(), camera->get_rayDirections(), n * 12, cudaMemcpyDeviceToHost);
    dump(out + ".rgba", rgba.data(), n * 16);
    dump(out + ".dirs", dirs.data(), n * 12);
    dump(out + ".brick", cpu.data(), nv * 4);
    delete rc; delete fm; delete camera;
    cudaFree(gpu); cudaFree(screen);
    return 0;
}

static int run_lru(int argc, char** argv) {
    if (argc < 11) die("lru: args");
    char* vol = argv[2];
    int nGPU = atoi(argv[3]), nCPU = atoi(argv[4]);
    int levelO = atoi(argv[5]), levelC = atoi(argv[6]), nLevels = atoi(argv[7]);
    int inc = atoi(argv[8]);
    FILE* f = fopen(argv[9], "rb");
    if (!f) die("seq open");
    int rounds = 0, m = 0;
    if (fread(&rounds, 4, 1, f) != 1 || fread(&m, 4, 1, f) != 1) die("seq header");
    int cd = 1 << (nLevels - levelC);
    lruCache* c = new lruCache(vol, (char*)"value", nGPU, make_int3(cd, cd, cd), inc, levelC, levelO, nCPU);
    std::vector<visibleCube_t> vc(m);
    std::vector<unsigned char> outb;
    for (int r = 0; r < rounds; r++) {
        for (int i = 0; i < m; i++) {
            unsigned long long id; unsigned char s;
            if (fread(&id, 8, 1, f) != 1 || fread(&s, 1, 1, f) != 1) die("seq body");
            vc[i].id = id; vc[i].state = s; vc[i].data = 0; vc[i].cubeID = 0;
        }
        c->updateCache(vc.data(), m, nLevels);
        for (int i = 0; i < m; i++) {
            int slot = vc[i].data ? (int)((vc[i].data - c->cacheData) / c->offsetCube) : -1;
            unsigned char s = vc[i].state;
            unsigned long long cid = vc[i].cubeID;
            const unsigned char* ps = (const unsigned char*)&slot;
            const unsigned char* pc = (const unsigned char*)&cid;
            outb.push_back(s);
            outb.insert(outb.end(), ps, ps + 4);
            outb.insert(outb.end(), pc, pc + 8);
        }
    }
    fclose(f);
    long long stats[5] = {c->access, c->hitsCPU, c->missCPU, c->hitsGPU, c->missGPU};
    dump(std::string(argv[10]), outb.data(), outb.size());
    dump(std::string(argv[10]) + ".stats", stats, sizeof(stats));
    delete c;
    return 0;
}

int main(int argc, char** argv) {
    if (argc < 2) die("usage");
    watchdog(240);
    std::string mode = argv[1];
    if (mode == "render") return run_render(argc, argv);
    if (mode == "cube") return run_cube(argc, argv);
    if (mode == "lru") return run_lru(argc, argv);
    die("unknown mode");
    return 1;
}
