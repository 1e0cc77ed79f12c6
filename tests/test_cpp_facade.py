"""The header-only C++ facade (include/visualtur.hpp) compiles against the
reference's call surface and links libvt.so: a program written like the
reference's src/testFileManager.cu runs its known-answer checks through
vt::FileManager, and camera operations through vt::Camera match the oracle
bit for bit."""
import os
import subprocess

import numpy as np
import pytest

import vt_fixtures as F
import visualtur_b200 as vt
from oracle import oracle as orc

PROG = r'''
#define VT_REFERENCE_NAMES
#include "visualtur.hpp"
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <vector>

static int3 mk(int x, int y, int z) { int3 r; r.x = x; r.y = y; r.z = z; return r; }
static float3 mkf(float x, float y, float z) { float3 r; r.x = x; r.y = y; r.z = z; return r; }

int main(int argc, char** argv) {
    FileManager fm(argv[1], "value");
    const int inc = 2, dim2 = 32 + 2 * inc;
    std::vector<float> d1(dim2 * dim2 * dim2), d2(dim2 * dim2 * dim2);
    fm.readHDF5_Voxel_Array(mk(0, 0, 0), mk(dim2, dim2, dim2), d1.data());
    int shifts[4][3] = {{-4, -4, -4}, {-4, 0, 0}, {0, -4, 0}, {0, 0, 0}};
    for (auto& sh : shifts) {           /* src/testFileManager.cu:62-100 */
        int3 mn = mk(sh[0], sh[1], sh[2]);
        int3 mx = mk(mn.x + dim2, mn.y + dim2, mn.z + dim2);
        fm.readHDF5_Voxel_Array(mn, mx, d2.data());
        for (int i = 0; i < dim2; i++) for (int j = 0; j < dim2; j++) for (int k = 0; k < dim2; k++) {
            float got = d2[k + j * dim2 + i * dim2 * dim2];
            int a = i + mn.x, b = j + mn.y, c = k + mn.z;
            float want = (a < 0 || b < 0 || c < 0) ? 0.0f : d1[c + b * dim2 + a * dim2 * dim2];
            if (a >= dim2 || b >= dim2 || c >= dim2) continue;
            if (got != want) { printf("KAT mismatch\n"); return 1; }
        }
    }
    Camera cam(1, 72, 80, 50.0f, 25.0f, 27.5f);
    cam.Move(mkf(31.5f, 31.5f, 181.5f)); cam.RotateY(10.0f); cam.RotateX(-8.0f); cam.RotateZ(5.0f);
    cam.MoveForward(20.0f); cam.StrafeRight(3.0f); cam.MoveUpward(-2.0f);
    float3 v[4] = {cam.get_look(), cam.get_up(), cam.get_right(), cam.get_position()};
    for (auto& x : v) printf("%08x %08x %08x\n", *(unsigned*)&x.x, *(unsigned*)&x.y, *(unsigned*)&x.z);
    float h = cam.get_h(), w = cam.get_w();
    printf("%08x %08x\n", *(unsigned*)&h, *(unsigned*)&w);
    try { Camera bad(2, 8, 8, 1.0f, 30.0f, 30.0f); return 2; } catch (const vt::Error& e) { printf("ok %d\n", e.status); }
    return 0;
}
'''


def test_cpp_facade_compiles_and_matches(workdir):
    src = os.path.join(workdir, "facade.cpp")
    exe = os.path.join(workdir, "facade")
    open(src, "w").write(PROG)
    inc = os.path.join(F.ROOT, "include")
    libdir = os.path.dirname(vt.LIB_PATH)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", inc, "-I", "/usr/local/cuda/include", src, "-o", exe,
                        "-L", libdir, "-lvt", "-Wl,-rpath," + libdir], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    raw = os.path.join(workdir, "facade.raw")
    F.write_raw(raw, F.case_volume("s64"))
    out = subprocess.run([exe, raw], capture_output=True, text=True)
    assert out.returncode == 0, out.stdout + out.stderr
    lines = out.stdout.split("\n")
    c = orc.Camera(72, 80, 50.0, 25.0, 27.5)
    orc.apply_ops(c, [("mv", (31.5, 31.5, 181.5)), ("ry", 10.0), ("rx", -8.0), ("rz", 5.0), ("mf", 20.0),
                      ("sr", 3.0), ("mu", -2.0)])
    st = c.state()
    hexf = lambda x: "%08x" % np.float32(x).view(np.uint32)
    want = [" ".join(hexf(a) for a in st[k]) for k in ("look", "up", "right", "position")]
    want.append("%s %s" % (hexf(st["h"]), hexf(st["w"])))
    assert lines[:5] == want
    assert lines[5] == "ok %d" % vt.VT_ERR_UNSUPPORTED


RENDER_PROG = r'''
#define VT_REFERENCE_NAMES
#include "visualtur.hpp"
#include <cuda_runtime.h>
#include <cstdio>
#include <vector>

/* shaped like src/testVisualTur.cu:28-110: parameters, a camera move, a
 * device pixel buffer, updateVisibleCubes, copy back, strafe, again */
int main(int argc, char** argv) {
    visualTurParams_t p;
    p.W = 96; p.H = 96; p.fov_H = 30.0f; p.fov_W = 30.0f; p.distance = 50.0f; p.numRayPx = 1;
    p.maxElementsCache = 512; p.maxElementsCache_CPU = 512;
    p.dimCubeCache.x = p.dimCubeCache.y = p.dimCubeCache.z = 8; p.cubeInc = 3; p.levelCubes = 3;
    p.hdf5File = argv[1]; p.dataset_name = (char*)"value"; p.octreeFile = argv[2]; p.octreeLevel = 4;
    visualTur* v = new visualTur(p);
    float3 mv; mv.x = 31.5f; mv.y = 31.5f; mv.z = 181.5f;
    v->camera_Move(mv);
    float* screenG = nullptr;
    if (cudaMalloc(&screenG, sizeof(float) * p.W * p.H * 4) != cudaSuccess) return 3;
    std::vector<float> screenC(p.W * p.H * 4);
    FILE* f = fopen(argv[3], "wb");
    for (int m = 0; m < 2; m++) {
        v->updateVisibleCubes(screenG);
        if (cudaMemcpy(screenC.data(), screenG, screenC.size() * 4, cudaMemcpyDeviceToHost) != cudaSuccess) return 4;
        fwrite(screenC.data(), 4, screenC.size(), f);
        v->camera_StrafeRight(0.5f);
    }
    fclose(f);
    cudaFree(screenG);
    delete v;
    printf("rendered\n");
    return 0;
}
'''


@pytest.mark.gpu
def test_cpp_facade_renders_like_the_reference_program(workdir, cuda):
    src = os.path.join(workdir, "facade_render.cpp")
    exe = os.path.join(workdir, "facade_render")
    open(src, "w").write(RENDER_PROG)
    inc = os.path.join(F.ROOT, "include")
    libdir = os.path.dirname(vt.LIB_PATH)
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", inc, "-I", "/usr/local/cuda/include", src, "-o", exe,
                        "-L", libdir, "-lvt", "-Wl,-rpath," + libdir, "-L", "/usr/local/cuda/lib64", "-lcudart"],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    c = F.CASES["s64"]
    vol = F.case_volume("s64")
    h5 = os.path.join(workdir, "facade_s64.h5")
    vt.FileManager.CreateFile(vol, h5)
    octf = F.case_octree("s64", workdir)
    out = os.path.join(workdir, "facade_frames.f32")
    run = subprocess.run([exe, h5, octf, out], capture_output=True, text=True)
    assert run.returncode == 0 and "rendered" in run.stdout, run.stdout + run.stderr
    got = np.fromfile(out, np.float32).reshape(2, c["W"] * c["H"], 4)
    cam = F.oracle_camera("s64")
    o = orc.Octree(octf)
    for m in range(2):
        want = orc.render(o, vol, cam, c["levelO"], c["levelC"], c["inc"])["rgba"]
        assert np.array_equal(got[m].view(np.uint32), want.view(np.uint32))
        cam.StrafeRight(0.5)
