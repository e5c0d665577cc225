// Geometry preprocessing on the GPU: surface normals, tangent frames and
// boundary typing of a voxel mask, byte-identical to the CPU path
// (dsmc_geometry_finish, which follows ComplexGeometry::calculate_normals,
// calculate_tangents and find_boundary_points, dsmc/complexgeometry.cpp:928-1063).
//
// The reference sweeps voxels in index order and empties, in place, solid
// voxels that have no normal but an empty neighbour, so a voxel can see
// removals made earlier in the sweep.  The GPU evaluates every voxel against
// the unmodified mask (one thread per voxel); the host then replays, in sweep
// order, only the voxels whose window can contain an earlier removal: the
// removal candidates and, transitively, the later voxels around each actual
// removal.  Every other voxel's window is unchanged at its turn in the sweep,
// so its GPU result is the sequential one.
//
// Tangent seeds come from one sequential ran1(-1) stream (three draws per
// voxel), drawn on the host; the Gram-Schmidt frame is built on the GPU.
// Built with -fmad=false: every float/double operation rounds as on the host.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <queue>
#include <string>
#include <vector>

#include "dsmc_b200.h"
#include "dsmc_internal.h"
#include "dsmc_layout.h"

namespace dsmc {
namespace {

struct Dims {
    int X, Y, Z, avg;
};

__host__ __device__ inline uint64_t lin(const Dims &d, int i, int j, int k) {
    return ((uint64_t)((i + d.X) % d.X) * d.Y + (uint64_t)((j + d.Y) % d.Y)) * d.Z + (uint64_t)((k + d.Z) % d.Z);
}

// One voxel of calculate_normals against mask m: writes the normal and
// returns whether the voxel is emptied.
__host__ __device__ inline bool normal_of(const Dims &d, const uint8_t *m, int i, int j, int k, float out[3]) {
    bool any_solid = false, all_solid = true;
    float n0 = 0.f, n1 = 0.f, n2 = 0.f;
    for (int di = -1; di <= 1; ++di)
        for (int dj = -1; dj <= 1; ++dj)
            for (int dk = -1; dk <= 1; ++dk) {
                const int s = m[lin(d, i + di, j + dj, k + dk)];
                if (s > 0) any_solid = true;
                if (s == 0) all_solid = false;
                n0 -= s * di;
                n1 -= s * dj;
                n2 -= s * dk;
            }
    const double norm_sq = n0 * n0 + n1 * n1 + n2 * n2;
    if (norm_sq > 0) {
        n0 = n1 = n2 = 0.f;
        for (int di = -d.avg; di <= d.avg; ++di)
            for (int dj = -d.avg; dj <= d.avg; ++dj)
                for (int dk = -d.avg; dk <= d.avg; ++dk) {
                    const int s = m[lin(d, i + di, j + dj, k + dk)];
                    n0 -= s * di;
                    n1 -= s * dj;
                    n2 -= s * dk;
                }
    }
    const double norm = (double)sqrtf(n0 * n0 + n1 * n1 + n2 * n2);
    bool emptied = false;
    if (norm > 0) {
        n0 = (float)(n0 / norm);
        n1 = (float)(n1 / norm);
        n2 = (float)(n2 / norm);
    } else if (!any_solid || !all_solid) {
        emptied = true;
    }
    out[0] = n0;
    out[1] = n1;
    out[2] = n2;
    return emptied;
}

__global__ void k_normals(Dims d, const uint8_t *mask, float *nrm, uint8_t *cand) {
    const uint64_t V = (uint64_t)d.X * d.Y * d.Z;
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < V;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const int k = (int)(idx % d.Z);
        const int j = (int)((idx / d.Z) % d.Y);
        const int i = (int)(idx / ((uint64_t)d.Y * d.Z));
        float n[3];
        const bool emptied = normal_of(d, mask, i, j, k, n);
        nrm[3 * idx] = n[0];
        nrm[3 * idx + 1] = n[1];
        nrm[3 * idx + 2] = n[2];
        // only a solid voxel changes when emptied
        cand[idx] = emptied && mask[idx] != 0;
    }
}

__global__ void k_frames(uint64_t V, const float *nrm, const float *seed, float *t1, float *t2, uint8_t *vox) {
    for (uint64_t idx = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; idx < V;
         idx += (uint64_t)gridDim.x * blockDim.x) {
        const float n0 = nrm[3 * idx], n1 = nrm[3 * idx + 1], n2 = nrm[3 * idx + 2];
        float a0 = seed[3 * idx], a1 = seed[3 * idx + 1], a2 = seed[3 * idx + 2];
        const double dot = n0 * a0 + n1 * a1 + n2 * a2;
        a0 = (float)(a0 - n0 * dot);
        a1 = (float)(a1 - n1 * dot);
        a2 = (float)(a2 - n2 * dot);
        double norm = (double)sqrtf(a0 * a0 + a1 * a1 + a2 * a2);
        if (norm > 0) {
            a0 = (float)(a0 / norm);
            a1 = (float)(a1 / norm);
            a2 = (float)(a2 / norm);
        }
        float b0 = a1 * n2 - a2 * n1;
        float b1 = a2 * n0 - a0 * n2;
        float b2 = a0 * n1 - a1 * n0;
        norm = (double)sqrtf(b0 * b0 + b1 * b1 + b2 * b2);
        if (norm > 0) {
            b0 = (float)(b0 / norm);
            b1 = (float)(b1 / norm);
            b2 = (float)(b2 / norm);
        }
        t1[3 * idx] = a0;
        t1[3 * idx + 1] = a1;
        t1[3 * idx + 2] = a2;
        t2[3 * idx] = b0;
        t2[3 * idx + 1] = b1;
        t2[3 * idx + 2] = b2;
        const double nn = n0 * n0 + n1 * n1 + n2 * n2;
        if (vox[idx] > 0 && nn > 0) vox[idx] = DSMC_VOX_BOUNDARY;
    }
}

}  // namespace
}  // namespace dsmc

using namespace dsmc;

namespace dsmc {
namespace {

// Device working buffers of the stencil: mask and candidate flags (V bytes
// each), normals, tangent seeds, tangents1, tangents2 (3 floats per voxel each).
struct StencilBuffers {
    uint8_t *mask, *cand;
    float *normals, *seed, *t1, *t2;
};

// The preprocessing itself, on buffers the caller provides: the normal
// stencil on the GPU, the sequential replay of the removals on the host, then
// the tangent frames and boundary typing on the GPU.  `what` prefixes error
// messages.  Allocates no device memory.
int finish_on_device(const Dims &d, uint8_t *vox, float *nrm, float *t1, float *t2, const StencilBuffers &b,
                     const char *what) {
    const uint64_t V = (uint64_t)d.X * d.Y * d.Z;
    auto cuda_err = [&](cudaError_t e) {
        set_thread_error(std::string(what) + ": " + cudaGetErrorString(e));
        return DSMC_ERR_CUDA;
    };
    cudaError_t e;
    if ((e = cudaMemcpy(b.mask, vox, V, cudaMemcpyHostToDevice))) return cuda_err(e);
    const int block = 256;
    const int grid = (int)std::min<uint64_t>((V + block - 1) / block, 148 * 64);
    k_normals<<<grid, block>>>(d, b.mask, b.normals, b.cand);
    if ((e = cudaGetLastError())) return cuda_err(e);
    std::vector<uint8_t> cand(V);
    if ((e = cudaMemcpy(nrm, b.normals, 12 * V, cudaMemcpyDeviceToHost)) ||
        (e = cudaMemcpy(cand.data(), b.cand, V, cudaMemcpyDeviceToHost)))
        return cuda_err(e);
    // Sequential replay of the voxels a removal can reach, in sweep order.
    std::priority_queue<uint64_t, std::vector<uint64_t>, std::greater<uint64_t>> dirty;
    std::vector<uint8_t> queued(V, 0);
    for (uint64_t idx = 0; idx < V; ++idx)
        if (cand[idx]) {
            dirty.push(idx);
            queued[idx] = 1;
        }
    const int reach = std::max(1, d.avg);
    while (!dirty.empty()) {
        const uint64_t idx = dirty.top();
        dirty.pop();
        const int k = (int)(idx % d.Z), j = (int)((idx / d.Z) % d.Y), i = (int)(idx / ((uint64_t)d.Y * d.Z));
        float n[3];
        const bool emptied = normal_of(d, vox, i, j, k, n);
        nrm[3 * idx] = n[0];
        nrm[3 * idx + 1] = n[1];
        nrm[3 * idx + 2] = n[2];
        if (emptied && vox[idx] != 0) {
            vox[idx] = 0;
            for (int di = -reach; di <= reach; ++di)
                for (int dj = -reach; dj <= reach; ++dj)
                    for (int dk = -reach; dk <= reach; ++dk) {
                        const uint64_t q = lin(d, i + di, j + dj, k + dk);
                        if (q > idx && !queued[q]) {
                            queued[q] = 1;
                            dirty.push(q);
                        }
                    }
        }
    }
    // Tangent seeds: ran1(-1), three per voxel in index order.
    std::vector<float> seed(3 * V);
    Ran1 rnd(-1);
    for (uint64_t q = 0; q < 3 * V; ++q) seed[q] = (float)rnd.next();
    if ((e = cudaMemcpy(b.normals, nrm, 12 * V, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(b.seed, seed.data(), 12 * V, cudaMemcpyHostToDevice)) ||
        (e = cudaMemcpy(b.mask, vox, V, cudaMemcpyHostToDevice)))
        return cuda_err(e);
    k_frames<<<grid, block>>>(V, b.normals, b.seed, b.t1, b.t2, b.mask);
    if ((e = cudaGetLastError())) return cuda_err(e);
    if ((e = cudaMemcpy(t1, b.t1, 12 * V, cudaMemcpyDeviceToHost)) ||
        (e = cudaMemcpy(t2, b.t2, 12 * V, cudaMemcpyDeviceToHost)) ||
        (e = cudaMemcpy(vox, b.mask, V, cudaMemcpyDeviceToHost)))
        return cuda_err(e);
    return DSMC_OK;
}

}  // namespace
}  // namespace dsmc

extern "C" int dsmc_geometry_finish_gpu(int device_id, uint32_t nx, uint32_t ny, uint32_t nz, int avg, uint8_t *vox,
                                        float *nrm, float *t1, float *t2) {
    if (!vox || !nrm || !t1 || !t2 || nx == 0 || ny == 0 || nz == 0 || avg < 0) return DSMC_ERR_ARG;
    if (cudaSetDevice(device_id) != cudaSuccess) {
        set_thread_error("no CUDA device for geometry preprocessing");
        return DSMC_ERR_NO_DEVICE;
    }
    const Dims d = {(int)nx, (int)ny, (int)nz, avg};
    const uint64_t V = (uint64_t)nx * ny * nz;
    StencilBuffers b = {};
    auto cleanup = [&]() {
        cudaFree(b.mask);
        cudaFree(b.cand);
        cudaFree(b.normals);
        cudaFree(b.seed);
        cudaFree(b.t1);
        cudaFree(b.t2);
    };
    cudaError_t e;
    if ((e = cudaMalloc(&b.mask, V)) || (e = cudaMalloc(&b.cand, V)) || (e = cudaMalloc(&b.normals, 12 * V)) ||
        (e = cudaMalloc(&b.seed, 12 * V)) || (e = cudaMalloc(&b.t1, 12 * V)) || (e = cudaMalloc(&b.t2, 12 * V))) {
        cleanup();
        set_thread_error(std::string("geometry on the GPU: ") + cudaGetErrorString(e));
        return DSMC_ERR_CUDA;
    }
    const int rc = finish_on_device(d, vox, nrm, t1, t2, b, "geometry on the GPU");
    cleanup();
    return rc;
}

// ---------------------------------------------------------------------------
// The same preprocessing for callers that cannot allocate device memory: a
// caller that runs where a cudaMalloc is not allowed or not wanted (inside a
// region whose device memory is fixed in advance, or where the implicit
// device synchronisation of an allocation would stall other work) still needs
// the stencil's device-side working buffers.  They live in this file-scope
// array instead, sized for grids of up to kNoAllocMaxVoxels voxels (64^3;
// 50 bytes per voxel, 13.1 MB that every GPU which loads this library keeps
// until the process exits).
//
// The array's host-side name is only a stand-in for the device symbol: the
// device address is looked up with cudaGetSymbolAddress once per device, on
// that device's first call, and cached.  That first call should therefore
// come before any stream capture.  A cudaDeviceReset by the caller unloads
// the module and invalidates the cached address: a process that resets a
// device must not call this entry point on that device afterwards.  Every call reuses the same array and
// leaves its contents behind; each kernel here rewrites every element it
// later reads, so nothing needs clearing between calls.  Calls that overlap
// on the GPU (two host threads, same device) race on the array.
namespace dsmc {
namespace {
constexpr uint64_t kNoAllocMaxVoxels = 64ull * 64ull * 64ull;
constexpr uint64_t kNoAllocBytes = kNoAllocMaxVoxels * (2 + 4 * 12);
constexpr int kNoAllocMaxDevices = 64;
static __device__ __align__(256) unsigned char g_geometry_scratch[kNoAllocBytes];

std::mutex g_scratch_mutex;
unsigned char *g_scratch_ptr[kNoAllocMaxDevices] = {};
}  // namespace
}  // namespace dsmc

extern "C" int dsmc_geometry_finish_gpu_noalloc(int device_id, uint32_t nx, uint32_t ny, uint32_t nz, int avg,
                                                uint8_t *vox, float *nrm, float *t1, float *t2) {
    if (!vox || !nrm || !t1 || !t2 || nx == 0 || ny == 0 || nz == 0 || avg < 0) return DSMC_ERR_ARG;
    const uint64_t V = (uint64_t)nx * ny * nz;
    if (V > kNoAllocMaxVoxels) {
        set_thread_error("dsmc_geometry_finish_gpu_noalloc: grid of " + std::to_string(V) +
                         " voxels exceeds the fixed scratch for " + std::to_string(kNoAllocMaxVoxels) +
                         " voxels (64^3); use dsmc_geometry_finish_gpu");
        return DSMC_ERR_CAPACITY;
    }
    if (device_id < 0 || device_id >= kNoAllocMaxDevices || cudaSetDevice(device_id) != cudaSuccess) {
        set_thread_error("no CUDA device for geometry preprocessing");
        return DSMC_ERR_NO_DEVICE;
    }
    unsigned char *base = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_ptr[device_id]) {
            void *p = nullptr;
            const cudaError_t e = cudaGetSymbolAddress(&p, g_geometry_scratch);
            if (e != cudaSuccess) {
                set_thread_error(std::string("dsmc_geometry_finish_gpu_noalloc: scratch address: ") +
                                 cudaGetErrorString(e));
                return DSMC_ERR_CUDA;
            }
            g_scratch_ptr[device_id] = static_cast<unsigned char *>(p);
        }
        base = g_scratch_ptr[device_id];
    }
    // layout: mask[V], cand[V], then normals, seeds, tangents1, tangents2
    // (3 floats per voxel each), every part 16-byte aligned
    StencilBuffers b;
    b.mask = base;
    b.cand = base + kNoAllocMaxVoxels;
    b.normals = reinterpret_cast<float *>(base + 2 * kNoAllocMaxVoxels);
    b.seed = b.normals + 3 * kNoAllocMaxVoxels;
    b.t1 = b.seed + 3 * kNoAllocMaxVoxels;
    b.t2 = b.t1 + 3 * kNoAllocMaxVoxels;
    const Dims d = {(int)nx, (int)ny, (int)nz, avg};
    return finish_on_device(d, vox, nrm, t1, t2, b, "geometry on the GPU (fixed scratch)");
}
