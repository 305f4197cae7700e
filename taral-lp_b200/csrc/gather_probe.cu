// gather_probe: the random-gather floor of the SpMV phases on this GPU. Times, with CUDA events and an L2 flush
// (256 MB write) before every launch, kernels over `count` nonzeros (int32 index + float value, 16-byte loads):
//   stream  -- the index and value arrays alone (no gather);
//   l2      -- plus one gathered float per nonzero at a uniform random index into an n-float vector (L2 sectors);
//   dsmem   -- the same gathers from the vector held in the distributed shared memory of a thread-block cluster
//              (16 CTAs x 128 KB; the slices are refilled from global memory in every launch, as a PDHG phase
//              would have to).
// Prints one JSON line per (n, kernel). Indices are generated in [0, n) on the host; every remote shared-memory
// read lies between the two cluster barriers of its launch.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

namespace cg = cooperative_groups;

#define PK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));              \
            std::exit(1);                                                              \
        }                                                                              \
    } while (0)

constexpr int kSlice = 32768;  // floats per CTA of the cluster (128 KB)
constexpr int kCluster = 16;

template <bool GATHER>
__global__ void __launch_bounds__(256) k_stream(int count, const int* __restrict__ idx, const float* __restrict__ val,
                                                const float* __restrict__ x, float* __restrict__ out) {
    float acc = 0.f;
    const int quads = count / 4;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += gridDim.x * blockDim.x) {
        const int4 c = reinterpret_cast<const int4*>(idx)[q];
        const float4 v = reinterpret_cast<const float4*>(val)[q];
        if (GATHER) acc += v.x * __ldg(x + c.x) + v.y * __ldg(x + c.y) + v.z * __ldg(x + c.z) + v.w * __ldg(x + c.w);
        else acc += v.x + v.y + v.z + v.w + float(c.x ^ c.w);
    }
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

__global__ void __launch_bounds__(512) k_dsmem(int count, const int* __restrict__ idx, const float* __restrict__ val,
                                               const float* __restrict__ x, int n, float* __restrict__ out) {
    extern __shared__ float slice[];
    __shared__ const float* base[kCluster];
    cg::cluster_group cl = cg::this_cluster();
    const int rank = int(cl.block_rank());
    for (int i = threadIdx.x; i < kSlice; i += blockDim.x) {
        const int g = rank * kSlice + i;
        slice[i] = g < n ? x[g] : 0.f;
    }
    if (threadIdx.x < kCluster) base[threadIdx.x] = cl.map_shared_rank(slice, int(threadIdx.x));
    cl.sync();
    float acc = 0.f;
    const int quads = count / 4;
    for (int q = blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += gridDim.x * blockDim.x) {
        const int4 c = reinterpret_cast<const int4*>(idx)[q];
        const float4 v = reinterpret_cast<const float4*>(val)[q];
        acc += v.x * base[c.x >> 15][c.x & (kSlice - 1)] + v.y * base[c.y >> 15][c.y & (kSlice - 1)] +
               v.z * base[c.z >> 15][c.z & (kSlice - 1)] + v.w * base[c.w >> 15][c.w & (kSlice - 1)];
    }
    cl.sync();
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;
}

template <class L>
static double time_us(L launch, float* flush, size_t flush_n, int reps) {
    cudaEvent_t a, b;
    PK(cudaEventCreate(&a));
    PK(cudaEventCreate(&b));
    for (int i = 0; i < 3; ++i) launch();
    PK(cudaGetLastError());
    PK(cudaDeviceSynchronize());
    double tot = 0;
    for (int r = 0; r < reps; ++r) {
        PK(cudaMemsetAsync(flush, r & 0xff, flush_n * sizeof(float)));
        PK(cudaEventRecord(a));
        launch();
        PK(cudaEventRecord(b));
        PK(cudaEventSynchronize(b));
        float ms = 0;
        PK(cudaEventElapsedTime(&ms, a, b));
        tot += ms;
    }
    PK(cudaGetLastError());
    cudaEventDestroy(a), cudaEventDestroy(b);
    return tot / reps * 1e3;
}

int main(int argc, char** argv) {
    const int count = argc > 1 ? std::atoi(argv[1]) / 4 * 4 : 5000000;
    const size_t flush_n = size_t(64) << 20;
    const int nmax = kCluster * kSlice;
    int sms = 0;
    PK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    int *d_idx;
    float *d_val, *d_x, *d_out, *flush;
    PK(cudaMalloc(&d_idx, size_t(count) * 4));
    PK(cudaMalloc(&d_val, size_t(count) * 4));
    PK(cudaMalloc(&d_x, size_t(nmax) * 4));
    PK(cudaMalloc(&d_out, size_t(sms) * 8 * 512 * 4));
    PK(cudaMalloc(&flush, flush_n * 4));
    PK(cudaMemset(d_val, 0, size_t(count) * 4));
    PK(cudaMemset(d_x, 0, size_t(nmax) * 4));
    PK(cudaFuncSetAttribute(k_dsmem, cudaFuncAttributeMaxDynamicSharedMemorySize, kSlice * 4));
    PK(cudaFuncSetAttribute(k_dsmem, cudaFuncAttributeNonPortableClusterSizeAllowed, 1));
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = kCluster, attr[0].val.clusterDim.y = 1, attr[0].val.clusterDim.z = 1;
    cudaLaunchConfig_t cfg = {};
    cfg.blockDim = dim3(512), cfg.dynamicSmemBytes = kSlice * 4, cfg.attrs = attr, cfg.numAttrs = 1;
    cfg.gridDim = dim3(kCluster);
    int clusters = 0;
    PK(cudaOccupancyMaxActiveClusters(&clusters, k_dsmem, &cfg));
    cfg.gridDim = dim3(kCluster * std::max(clusters, 1));
    std::mt19937 rng(1);
    for (int n : {500000, 200000}) {
        std::vector<int> h(count);
        std::uniform_int_distribution<int> U(0, n - 1);
        for (int& v : h) v = U(rng);
        PK(cudaMemcpy(d_idx, h.data(), size_t(count) * 4, cudaMemcpyHostToDevice));
        const int grid = sms * 8;
        const double t_stream = time_us([&] { k_stream<false><<<grid, 256>>>(count, d_idx, d_val, d_x, d_out); }, flush, flush_n, 10);
        const double t_l2 = time_us([&] { k_stream<true><<<grid, 256>>>(count, d_idx, d_val, d_x, d_out); }, flush, flush_n, 10);
        double t_ds = -1;
        if (clusters > 0)
            t_ds = time_us([&] { PK(cudaLaunchKernelEx(&cfg, k_dsmem, count, (const int*)d_idx, (const float*)d_val,
                                                       (const float*)d_x, n, d_out)); }, flush, flush_n, 10);
        std::printf("{\"n\": %d, \"nonzeros\": %d, \"stream_us\": %.2f, \"stream_gbs\": %.0f, \"l2_gather_us\": %.2f, "
                    "\"l2_gathers_per_s\": %.4g, \"dsmem_gather_us\": %.2f, \"dsmem_gathers_per_s\": %.4g, "
                    "\"dsmem_clusters\": %d}\n", n, count, t_stream, 8.0 * count / t_stream / 1e3, t_l2,
                    count / t_l2 * 1e6, t_ds, t_ds > 0 ? count / t_ds * 1e6 : 0.0, clusters);
    }
    return 0;
}
