// KKT evaluation that allocates no device memory (include/taral_pdhg.h, taral_kkt_eval_noalloc).
//
// Some callers cannot call cudaMalloc: a host whose device memory is reserved up front by another allocator
// (a framework's caching allocator that owns the whole GPU), or a solve loop that must not pay cudaMalloc's
// implicit device synchronisation between iterations. For them this entry point runs the same reduction kernels
// as pdhg_eval (k_eval_row / k_eval_col, fixed grid, fixed-order finish) on vectors the caller already holds,
// with its scratch -- the per-CTA partial sums and the two completion tickets -- in the file-scope array below
// instead of in memory allocated per context. The caller passes every input and the output buffer.
#include <cuda_runtime.h>

#include <climits>
#include <mutex>

#include "../../include/taral_pdhg.h"
#include "kernels.cuh"

namespace {

constexpr int kNoAllocBlocks = 296;                          // CTAs per reduction, as pdhg_eval uses
constexpr int kScratchDoubles = 2 * kNoAllocBlocks * 5 + 2;  // row partials, column partials, 2 tickets (16 B)
// Every GPU that loads the library holds these 23,696 bytes until the process exits.
static __device__ __align__(256) double g_kkt_scratch[kScratchDoubles];

constexpr int kMaxDevices = 64;
double* g_scratch_addr[kMaxDevices] = {};  // device address of g_kkt_scratch, per device, set on first use
std::mutex g_setup;

int reduction_grid(int k) { return k <= 0 ? 1 : (k + 255) / 256 < kNoAllocBlocks ? (k + 255) / 256 : kNoAllocBlocks; }

template <class T>
int launch(int m, int n, double f, const void* Ax, const void* z, const void* rl, const void* ru, const void* Dr,
           const void* zlast, const void* x, const void* ATz, const void* c, const void* l, const void* u,
           const void* Dc, const void* xlast, double* out, double* scratch, cudaStream_t s) {
    using namespace taral;
    unsigned* tickets = reinterpret_cast<unsigned*>(scratch + 2 * kNoAllocBlocks * 5);
    // The tickets must start at zero; a call that was interrupted could have left them set.
    if (cudaMemsetAsync(tickets, 0, 2 * sizeof(unsigned), s) != cudaSuccess) return TARAL_ERR_CUDA;
    k_eval_row<T, T><<<reduction_grid(m), kRedThreads, 0, s>>>(
        m, f, static_cast<const T*>(Ax), static_cast<const T*>(z), static_cast<const T*>(rl),
        static_cast<const T*>(ru), static_cast<const T*>(Dr), static_cast<const T*>(zlast), scratch, tickets, out);
    k_eval_col<T, T><<<reduction_grid(n), kRedThreads, 0, s>>>(
        n, f, static_cast<const T*>(x), static_cast<const T*>(ATz), static_cast<const T*>(c),
        static_cast<const T*>(l), static_cast<const T*>(u), static_cast<const T*>(Dc), static_cast<const T*>(xlast),
        scratch + kNoAllocBlocks * 5, tickets + 1, out + 5);
    return cudaGetLastError() == cudaSuccess ? TARAL_OK : TARAL_ERR_CUDA;
}

}  // namespace

extern "C" int taral_kkt_eval_noalloc(int m, int n, int dtype, double f, const void* Ax, const void* z,
                                      const void* rl, const void* ru, const void* Dr, const void* zlast,
                                      const void* x, const void* ATz, const void* c, const void* l, const void* u,
                                      const void* Dc, const void* xlast, double* out10, void* stream) {
    if (m < 0 || n < 0 || m > TARAL_NOALLOC_MAX_DIM || n > TARAL_NOALLOC_MAX_DIM) return TARAL_ERR_INPUT;
    if (dtype != TARAL_FP64 && dtype != TARAL_FP32) return TARAL_ERR_INPUT;
    if (!out10) return TARAL_ERR_INPUT;
    if (m && (!Ax || !z || !rl || !ru || !Dr || !zlast)) return TARAL_ERR_INPUT;
    if (n && (!x || !ATz || !c || !l || !u || !Dc || !xlast)) return TARAL_ERR_INPUT;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return TARAL_ERR_NO_DEVICE;
    if (dev < 0 || dev >= kMaxDevices) return TARAL_ERR_INPUT;
    double* scratch;
    {
        // Set-up, once per device, with that device current: the host-side name g_kkt_scratch is not a device
        // address, so the kernels get the address the runtime reports for this device.
        std::lock_guard<std::mutex> lock(g_setup);
        if (!g_scratch_addr[dev]) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_kkt_scratch) != cudaSuccess || !p) return TARAL_ERR_CUDA;
            g_scratch_addr[dev] = static_cast<double*>(p);
        }
        scratch = g_scratch_addr[dev];
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (dtype == TARAL_FP32)
        return launch<float>(m, n, f, Ax, z, rl, ru, Dr, zlast, x, ATz, c, l, u, Dc, xlast, out10, scratch, s);
    return launch<double>(m, n, f, Ax, z, rl, ru, Dr, zlast, x, ATz, c, l, u, Dc, xlast, out10, scratch, s);
}
