// ORACLE - test infrastructure, not product code.
//
// Harness that runs the reference's own CUDA integrator on the GPU: it includes
// src/renderers/path_tracer.cu from the reference tree (for its file-static renderInit and
// renderKernel) and links the reference's world, primitive, material, camera, transform,
// distribution, material-lookup and framebuffer sources, all compiled with nvcc for sm_100a
// by `make -C oracle refbench` into oracle/_ref/librefbench.so (and a -fmad=false build,
// librefbench_nofma.so). Nothing of the reference is copied into this repository.
//
// Scene upload follows CUDAGlobals (src/cuda_globals.cu:10-139) and
// MaterialLookup::copyMaterials (src/materials/material_lookup.cu:13-123); the environment
// light follows EnvironmentLightParams::createEnvironmentLight
// (src/lights/environment_light.cu:14-56) with the map passed in memory instead of loaded
// from an EXR file. Frames are launched as PathTracer::renderAsync does
// (src/renderers/path_tracer.cu:285-336): renderKernel on 16x16 blocks, then
// updateFramebuffer, timed with CUDA events.
#include <cfloat>
#include <cstdio>
#include <memory>
#include <vector>

#include "renderers/path_tracer.cu"

using namespace rays;

namespace {

struct RefBench {
    int width = 0, height = 0;
    SceneData scene;
    MaterialLookup lookup{};
    MaterialLookup* d_lookup = nullptr;
    EnvironmentLight env = EnvironmentLight::None();
    EnvironmentLight* d_env = nullptr;
    Triangle* d_tris = nullptr;
    Sphere* d_sphs = nullptr;
    LightIndex* d_lights = nullptr;
    World* d_world = nullptr;
    Camera* d_camera = nullptr;
    float* d_env_data = nullptr;
    curandState* d_rand = nullptr;
    Vec3* d_pass = nullptr;
    Vec3* d_radiance = nullptr;
    uchar4* d_fb = nullptr;
    int currentSamples = 0;
};

__global__ void initWorld(World* world, Triangle* t, int nt, Sphere* s, int ns, LightIndex* l, int nl,
                          EnvironmentLight* env, MaterialLookup* lookup) {
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    *world = World(t, nt, s, ns, l, nl, env, lookup);
}

__global__ void hitKernel(const World* world, const float* o, const float* d, const float* tmin, const float* tmax,
                          int n, int* type, int* id, int* mat, float* t) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const Ray ray(Vec3(o[3 * i], o[3 * i + 1], o[3 * i + 2]), Vec3(d[3 * i], d[3 * i + 1], d[3 * i + 2]));
    HitRecord rec;
    if (world->hit(ray, tmin[i], tmax[i], rec)) {
        type[i] = rec.index.primitiveType == PrimitiveType::Triangle ? 0 : 1;
        id[i] = rec.index.index;
        mat[i] = rec.materialID;
        t[i] = rec.t;
    } else {
        type[i] = -1;
        id[i] = -1;
        mat[i] = -1;
        t[i] = 0.f;
    }
}

int check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        fprintf(stderr, "refbench: %s: %s\n", what, cudaGetErrorString(e));
        return -1;
    }
    return 0;
}

}  // namespace

extern "C" {

void* refbench_create(int ntri, const float* tri_p, const float* tri_n, const int* tri_mat, int nsph, const float* sph,
                      const int* sph_mat, int nmat, const int* mtype, const float* albedo, const float* emit,
                      const float* ior, const float* alpha, int env_w, int env_h, const float* env_rgba) {
    RefBench* b = new RefBench();
    SceneData& sd = b->scene;
    for (int i = 0; i < ntri; i++) {
        const float* p = tri_p + (size_t)i * 9;
        const float* n = tri_n + (size_t)i * 9;
        sd.triangles.push_back(Triangle(Vec3(p[0], p[1], p[2]), Vec3(p[3], p[4], p[5]), Vec3(p[6], p[7], p[8]),
                                        Vec3(n[0], n[1], n[2]), Vec3(n[3], n[4], n[5]), Vec3(n[6], n[7], n[8]),
                                        tri_mat[i]));
    }
    for (int i = 0; i < nsph; i++) {
        const float* q = sph + (size_t)i * 4;
        sd.spheres.push_back(Sphere(Vec3(q[0], q[1], q[2]), q[3], sph_mat[i]));
    }
    for (int i = 0; i < nmat; i++) {
        switch (mtype[i]) {
            case 0:
                sd.materialParams.push_back(std::make_unique<LambertianParams>(
                    Vec3(albedo[3 * i], albedo[3 * i + 1], albedo[3 * i + 2]),
                    Vec3(emit[3 * i], emit[3 * i + 1], emit[3 * i + 2])));
                break;
            case 1: sd.materialParams.push_back(std::make_unique<MirrorParams>()); break;
            case 2: sd.materialParams.push_back(std::make_unique<GlassParams>(ior[i])); break;
            default: sd.materialParams.push_back(std::make_unique<MicrofacetParams>(alpha[i]));
        }
    }
    // emitter list (src/scene_data.cu:92-115)
    for (int i = 0; i < ntri; i++)
        if (sd.isEmitter(tri_mat[i])) sd.lightIndices.push_back({PrimitiveType::Triangle, i});
    for (int i = 0; i < nsph; i++)
        if (sd.isEmitter(sph_mat[i])) sd.lightIndices.push_back({PrimitiveType::Sphere, i});

    if (check(cudaMalloc((void**)&b->d_lookup, sizeof(MaterialLookup)), "malloc")) return nullptr;
    b->lookup.mallocMaterials(sd);
    b->lookup.copyMaterials(sd);
    if (check(cudaMemcpy(b->d_lookup, &b->lookup, sizeof(MaterialLookup), cudaMemcpyHostToDevice), "copy")) return nullptr;
    if (env_rgba && env_w > 0) {
        const size_t bytes = (size_t)env_w * env_h * 4 * sizeof(float);
        if (check(cudaMalloc((void**)&b->d_env_data, bytes), "malloc env")) return nullptr;
        if (check(cudaMemcpy(b->d_env_data, env_rgba, bytes, cudaMemcpyHostToDevice), "copy env")) return nullptr;
        std::vector<float> inten((size_t)env_w * env_h);
        for (int i = 0; i < env_w * env_h; i++)
            inten[i] = env_rgba[i * 4 + 0] + env_rgba[i * 4 + 1] + env_rgba[i * 4 + 2];
        PhiThetaDistributionBuilder builder(inten.data(), env_w, env_h);
        b->env = EnvironmentLight(b->d_env_data, builder.buildPhiThetaDistribution(), env_w, env_h);
    }
    const size_t nt = sd.triangles.size(), ns = sd.spheres.size(), nl = sd.lightIndices.size();
    if (check(cudaMalloc((void**)&b->d_tris, nt * sizeof(Triangle) + 16), "malloc")) return nullptr;
    if (check(cudaMalloc((void**)&b->d_sphs, ns * sizeof(Sphere) + 16), "malloc")) return nullptr;
    if (check(cudaMalloc((void**)&b->d_lights, nl * sizeof(LightIndex) + 16), "malloc")) return nullptr;
    if (check(cudaMalloc((void**)&b->d_env, sizeof(EnvironmentLight)), "malloc")) return nullptr;
    if (check(cudaMalloc((void**)&b->d_world, sizeof(World)), "malloc")) return nullptr;
    if (nt) cudaMemcpy(b->d_tris, sd.triangles.data(), nt * sizeof(Triangle), cudaMemcpyHostToDevice);
    if (ns) cudaMemcpy(b->d_sphs, sd.spheres.data(), ns * sizeof(Sphere), cudaMemcpyHostToDevice);
    if (nl) cudaMemcpy(b->d_lights, sd.lightIndices.data(), nl * sizeof(LightIndex), cudaMemcpyHostToDevice);
    cudaMemcpy(b->d_env, &b->env, sizeof(EnvironmentLight), cudaMemcpyHostToDevice);
    initWorld<<<1, 1>>>(b->d_world, b->d_tris, (int)nt, b->d_sphs, (int)ns, b->d_lights, (int)nl, b->d_env, b->d_lookup);
    if (check(cudaDeviceSynchronize(), "init world")) return nullptr;
    return b;
}

// Camera (src/core/camera.cu:5-21) + curand states (renderInit, path_tracer.cu:266-283).
int refbench_init(void* p, const float* cam, int width, int height) {
    RefBench* b = static_cast<RefBench*>(p);
    b->width = width;
    b->height = height;
    Camera c(Vec3(cam[0], cam[1], cam[2]), Vec3(cam[3], cam[4], cam[5]), Vec3(cam[6], cam[7], cam[8]), cam[9],
             Resolution{width, height}, cam[10] != 0.f);
    const size_t np = (size_t)width * height;
    if (check(cudaMalloc((void**)&b->d_camera, sizeof(Camera)), "malloc")) return -1;
    cudaMemcpy(b->d_camera, &c, sizeof(Camera), cudaMemcpyHostToDevice);
    if (check(cudaMalloc((void**)&b->d_rand, np * sizeof(curandState)), "malloc")) return -1;
    if (check(cudaMalloc((void**)&b->d_pass, np * sizeof(Vec3)), "malloc")) return -1;
    if (check(cudaMalloc((void**)&b->d_radiance, np * sizeof(Vec3)), "malloc")) return -1;
    if (check(cudaMalloc((void**)&b->d_fb, np * sizeof(uchar4)), "malloc")) return -1;
    renderInit<<<dim3(width, height), 1>>>(width, height, b->d_rand);
    b->currentSamples = 0;
    return check(cudaDeviceSynchronize(), "renderInit");
}

// One frame as PathTracer::renderAsync + pollRender. ms: device time of the frame.
int refbench_render(void* p, int spp, int maxDepth, int nee, float* ms) {
    RefBench* b = static_cast<RefBench*>(p);
    const dim3 blocks(b->width / 16 + 1, b->height / 16 + 1);
    const dim3 threads(16, 16);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0);
    renderKernel<<<blocks, threads>>>(b->d_pass, b->width, b->height, b->d_rand, b->d_world, b->d_camera, maxDepth, spp,
                                      nee != 0);
    updateFramebuffer(b->d_fb, b->d_pass, b->d_radiance, spp, b->currentSamples, b->width, b->height, 0);
    cudaEventRecord(e1);
    if (check(cudaEventSynchronize(e1), "frame")) return -1;
    if (check(cudaGetLastError(), "frame launch")) return -1;
    cudaEventElapsedTime(ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    b->currentSamples += spp;
    return 0;
}

// Running-mean radiance (Renderer::getRadianceBuffer, renderer.cpp:20-42): 3 floats per pixel.
int refbench_readback(void* p, float* rgb) {
    RefBench* b = static_cast<RefBench*>(p);
    return check(cudaMemcpy(rgb, b->d_radiance, (size_t)b->width * b->height * sizeof(Vec3), cudaMemcpyDeviceToHost),
                 "readback");
}

// World::hit on n rays (host arrays).
int refbench_trace(void* p, const float* o, const float* d, const float* tmin, const float* tmax, int n, int* type,
                   int* id, int* mat, float* t) {
    RefBench* b = static_cast<RefBench*>(p);
    float* buf = nullptr;
    const size_t N = (size_t)n;
    if (check(cudaMalloc((void**)&buf, N * 4 * 12), "malloc")) return -1;
    float *dO = buf, *dD = dO + 3 * N, *dMin = dD + 3 * N, *dMax = dMin + N;
    int *dT = (int*)(dMax + N), *dI = dT + N, *dM = dI + N;
    float* dt = (float*)(dM + N);
    cudaMemcpy(dO, o, 12 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(dD, d, 12 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(dMin, tmin, 4 * N, cudaMemcpyHostToDevice);
    cudaMemcpy(dMax, tmax, 4 * N, cudaMemcpyHostToDevice);
    hitKernel<<<(n + 127) / 128, 128>>>(b->d_world, dO, dD, dMin, dMax, n, dT, dI, dM, dt);
    int rc = check(cudaDeviceSynchronize(), "hit kernel");
    cudaMemcpy(type, dT, 4 * N, cudaMemcpyDeviceToHost);
    cudaMemcpy(id, dI, 4 * N, cudaMemcpyDeviceToHost);
    cudaMemcpy(mat, dM, 4 * N, cudaMemcpyDeviceToHost);
    cudaMemcpy(t, dt, 4 * N, cudaMemcpyDeviceToHost);
    cudaFree(buf);
    return rc;
}

void refbench_destroy(void* p) {
    RefBench* b = static_cast<RefBench*>(p);
    cudaFree(b->d_tris);
    cudaFree(b->d_sphs);
    cudaFree(b->d_lights);
    cudaFree(b->d_env);
    cudaFree(b->d_world);
    cudaFree(b->d_camera);
    cudaFree(b->d_rand);
    cudaFree(b->d_pass);
    cudaFree(b->d_radiance);
    cudaFree(b->d_fb);
    cudaFree(b->d_env_data);
    cudaFree(b->d_lookup);
    b->lookup.freeMaterials();
    delete b;
}

}  // extern "C"
