// gather_floor: the random-gather floor of the SpMV phases on this GPU, a measurement tool the benchmark runs beside
// the solve (not part of the library). With CUDA events and a 256 MB L2 flush before every launch it times two
// kernels over `count` nonzeros (int32 index + float value, 16-byte loads, a grid of 8 CTAs of 256 per SM):
//   stream -- the index and value arrays alone (no gather);
//   l2     -- the same stream plus one gathered float per nonzero at a uniformly random index into an n-float vector
//             (each gather costs one 32-byte L2 sector).
// Prints one JSON line per vector length n (500,000 and 200,000: the lengths of x and z of the benchmark LP).
// Indices are drawn in [0, n) on the host, so every gather stays inside the n-float vector.
#include <cuda_runtime.h>

#include <cstdio>
#include <cstdlib>
#include <random>
#include <vector>

#define PK(x)                                                                          \
    do {                                                                               \
        cudaError_t e_ = (x);                                                          \
        if (e_ != cudaSuccess) {                                                       \
            std::fprintf(stderr, "%s: %s\n", #x, cudaGetErrorString(e_));              \
            std::exit(1);                                                              \
        }                                                                              \
    } while (0)

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
    out[blockIdx.x * blockDim.x + threadIdx.x] = acc;  // keeps the loads live
}

template <class L>
static double time_us(L launch, void* flush, size_t flush_bytes, int reps) {
    cudaEvent_t a, b;
    PK(cudaEventCreate(&a));
    PK(cudaEventCreate(&b));
    for (int i = 0; i < 3; ++i) launch();
    PK(cudaGetLastError());
    PK(cudaDeviceSynchronize());
    double total_ms = 0;
    for (int r = 0; r < reps; ++r) {
        PK(cudaMemsetAsync(flush, r & 0xff, flush_bytes));
        PK(cudaEventRecord(a));
        launch();
        PK(cudaEventRecord(b));
        PK(cudaEventSynchronize(b));
        float ms = 0;
        PK(cudaEventElapsedTime(&ms, a, b));
        total_ms += ms;
    }
    PK(cudaGetLastError());
    cudaEventDestroy(a), cudaEventDestroy(b);
    return total_ms / reps * 1e3;
}

int main(int argc, char** argv) {
    const int count = argc > 1 ? std::atoi(argv[1]) / 4 * 4 : 5000000;
    const size_t flush_bytes = size_t(256) << 20;
    const int nmax = 500000;
    int sms = 0;
    PK(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
    const int grid = sms * 8;
    int* d_idx;
    float *d_val, *d_x, *d_out;
    void* flush;
    PK(cudaMalloc(&d_idx, size_t(count) * 4));
    PK(cudaMalloc(&d_val, size_t(count) * 4));
    PK(cudaMalloc(&d_x, size_t(nmax) * 4));
    PK(cudaMalloc(&d_out, size_t(grid) * 256 * 4));
    PK(cudaMalloc(&flush, flush_bytes));
    PK(cudaMemset(d_val, 0, size_t(count) * 4));
    PK(cudaMemset(d_x, 0, size_t(nmax) * 4));
    std::mt19937 rng(1);
    for (int n : {500000, 200000}) {
        std::vector<int> h(static_cast<size_t>(count));
        std::uniform_int_distribution<int> U(0, n - 1);
        for (int& v : h) v = U(rng);
        PK(cudaMemcpy(d_idx, h.data(), size_t(count) * 4, cudaMemcpyHostToDevice));
        const double t_stream =
            time_us([&] { k_stream<false><<<grid, 256>>>(count, d_idx, d_val, d_x, d_out); }, flush, flush_bytes, 10);
        const double t_l2 =
            time_us([&] { k_stream<true><<<grid, 256>>>(count, d_idx, d_val, d_x, d_out); }, flush, flush_bytes, 10);
        std::printf("{\"n\": %d, \"nonzeros\": %d, \"stream_us\": %.2f, \"stream_gbs\": %.0f, \"l2_gather_us\": %.2f, "
                    "\"l2_gathers_per_s\": %.4g}\n",
                    n, count, t_stream, 8.0 * count / t_stream / 1e3, t_l2, count / t_l2 * 1e6);
    }
    return 0;
}
