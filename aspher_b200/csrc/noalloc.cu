// Allocation-free periodic operator apply.
//
// Some callers cannot let a library allocate device memory: real-time loops
// that must never block in the allocator (cudaMalloc and cudaFree can
// synchronise the device), host applications that hand all of the GPU's
// memory to their own allocator up front, where a library cudaMalloc fails
// or fragments that pool, and plugins whose host process accounts for every
// device byte and forbids per-handle buffers.  aspher_periodic_matvec_noalloc
// serves them: the same doubly periodic apply as aspher_op_matvec on a
// PERIODIC operator, but with its half-spectrum scratch and twiddle tables in
// file-scope __device__ arrays, and no operator handle (the symbol
// scale/|m| is computed on the fly).  The caller passes only the input and
// the output.
//
// Limits and contract:
//   - grid_size is a power of two in [16, kNoAllocMaxNs] (1024); larger grids
//     are rejected (the static scratch is sized for 1024: (512+16) x 1024
//     double2 = 8.65 MB; the FP32 path uses the same array);
//   - the 8.65 MB are device memory of this file's module: with CUDA's lazy
//     module loading (the default since CUDA 12.2) the driver allocates them
//     when the module is first used on a device, i.e. in the first call on
//     that device, and holds them until the process exits.  A host whose
//     allocator reserves the GPU's memory up front should make the first
//     call before it reserves its pool (or run with CUDA_MODULE_LOADING=EAGER,
//     which loads the module with the library);
//   - the first call on a device sets that device up (symbol addresses, the
//     twiddle tables filled by a kernel on the caller's stream, the kernels'
//     shared-memory attributes per precision and size on their first use);
//     make that first call before any stream capture;
//   - `stream` must belong to the current device;
//   - every call shares the one scratch array, which keeps the last call's
//     contents: calls that overlap on the GPU (different streams, or
//     different host threads without ordering) race on it.  Nothing in the
//     scratch has to start at zero: every entry a call reads, it first writes.
#include "../../include/aspher_b200.h"
#include "functors.cuh"
#include "ops.hpp"

#include <atomic>
#include <cmath>
#include <mutex>

namespace asb {
namespace {

constexpr int kNoAllocMaxNs = 1024;
constexpr size_t kNoAllocSpecElems = (size_t)(kNoAllocMaxNs / 2 + 16) * kNoAllocMaxNs;
constexpr int kNoAllocTw = 2 * kNoAllocMaxNs;  // tables for L = 1..1024 at offset L

static __device__ __align__(256) double2 g_na_spec[kNoAllocSpecElems];
static __device__ __align__(256) double2 g_na_tw_d[kNoAllocTw];
static __device__ __align__(256) float2 g_na_tw_f[kNoAllocTw];

struct NaDevice {
    bool ready = false;
    void* spec = nullptr;
    double2* twd = nullptr;
    float2* twf = nullptr;
    // kernel attributes set, one bit per (precision, log2 grid_size)
    std::atomic<unsigned> attrs{0};
};
NaDevice g_na[64];
std::mutex g_na_mu;

// exp(-2 pi i k / L) for every power of two L <= kNoAllocMaxNs, at offset L
__global__ void k_na_twiddles() {
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kNoAllocTw;
         i += gridDim.x * blockDim.x) {
        if (i < 1) continue;
        int L = 1;
        while (2 * L <= i) L <<= 1;  // i in [L, 2L)
        const int k = i - L;
        double s, c;
        sincospi(-2.0 * (double)k / (double)L, &s, &c);
        g_na_tw_d[i] = make_double2(c, s);
        g_na_tw_f[i] = make_float2((float)c, (float)s);
    }
}

NaDevice& na_setup(cudaStream_t s) {
    int dev = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(ASPHER_ECUDA, "device index out of range");
    std::lock_guard<std::mutex> lk(g_na_mu);
    NaDevice& d = g_na[dev];
    if (d.ready) return d;
    // host code names the arrays only through their device addresses
    ASB_CUDA(cudaGetSymbolAddress(&d.spec, g_na_spec));
    ASB_CUDA(cudaGetSymbolAddress((void**)&d.twd, g_na_tw_d));
    ASB_CUDA(cudaGetSymbolAddress((void**)&d.twf, g_na_tw_f));
    k_na_twiddles<<<8, 256, 0, s>>>();
    ASB_CUDA(cudaGetLastError());
    ASB_CUDA(cudaStreamSynchronize(s));
    d.ready = true;
    return d;
}

void na_attr(const void* func, int bytes) {
    if (bytes > 48 * 1024)
        ASB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

// The three kernels of one periodic apply with launch variant 0 (the same
// kernels and layout as the operator path).
template <typename T, int NS>
struct NaKernels {
    static constexpr int LR = NS / 2, LC = NS, V = 0;
    static constexpr auto fwd = row_fwd_kernel<T, LR, false, V, LoadRealRows<T>, StoreTiled<T>>;
    static constexpr auto col = col_kernel<T, LC, LR, false, V, PeriodicMult<T>>;
    static constexpr auto inv = row_inv_kernel<T, LR, false, V, LoadTiled<T>, StoreRealRows<T>>;
    static constexpr int sm_fwd = row_fwd_smem<T, LR, false, V, LoadRealRows<T>>();
    static constexpr int sm_col = col_smem_total<T, LC, LR, false, V>();
    static constexpr int sm_inv = row_inv_smem<T, LR, false, V, LoadTiled<T>>();
    // their shared-memory attributes, set once per device, precision and size
    static void prepare(NaDevice& d) {
        const unsigned bit = 1u << ((sizeof(T) == 8 ? 16 : 0) + ilog2c(NS));
        if (d.attrs.load(std::memory_order_acquire) & bit) return;
        std::lock_guard<std::mutex> lk(g_na_mu);
        if (d.attrs.load(std::memory_order_relaxed) & bit) return;
        na_attr((const void*)fwd, sm_fwd);
        na_attr((const void*)col, sm_col);
        na_attr((const void*)inv, sm_inv);
        d.attrs.fetch_or(bit, std::memory_order_release);
    }
};

// One periodic apply: the static scratch and the static twiddles.
template <typename T, int NS>
void na_apply(NaDevice& d, double scale, const T* x, T* y, cudaStream_t s) {
    using K = NaKernels<T, NS>;
    constexpr int LR = K::LR, LC = K::LC, V = K::V;
    constexpr int ct = col_ct_v<T>(LC, LR, V);
    K::prepare(d);
    const cplx<T>* tw = reinterpret_cast<const cplx<T>*>(
        sizeof(T) == 8 ? (const void*)d.twd : (const void*)d.twf);
    cplx<T>* spec = static_cast<cplx<T>*>(d.spec);
    {
        constexpr int rb = row_rb_v<T>(LR, V), thr = row_threads<T>(LR, V);
        K::fwd<<<(NS + rb - 1) / rb, thr, K::sm_fwd, s>>>(
            LoadRealRows<T>{x, NS}, StoreTiled<T>{spec, NS, ct}, NS, tw + LR, tw + 2 * LR,
            nullptr);
    }
    {
        constexpr int thr = col_threads<T>(LC, LR, V);
        K::col<<<LR / ct + 1, thr, K::sm_col, s>>>(spec, NS, PeriodicMult<T>{scale, NS}, tw + LC,
                                                   nullptr);
    }
    {
        constexpr int rb = row_rb_v<T>(LR, V), thr = row_threads<T>(LR, V);
        K::inv<<<(NS + rb - 1) / rb, thr, K::sm_inv, s>>>(
            LoadTiled<T>{spec, NS, ct}, StoreRealRows<T>{y, NS}, NS, tw + LR, tw + 2 * LR,
            nullptr);
    }
    count_launches(3);
    ASB_CUDA(cudaGetLastError());
}

template <typename T>
void na_dispatch(int Ns, NaDevice& d, double scale, const T* x, T* y, cudaStream_t s) {
    switch (Ns) {
        case 16: na_apply<T, 16>(d, scale, x, y, s); break;
        case 32: na_apply<T, 32>(d, scale, x, y, s); break;
        case 64: na_apply<T, 64>(d, scale, x, y, s); break;
        case 128: na_apply<T, 128>(d, scale, x, y, s); break;
        case 256: na_apply<T, 256>(d, scale, x, y, s); break;
        case 512: na_apply<T, 512>(d, scale, x, y, s); break;
        case 1024: na_apply<T, 1024>(d, scale, x, y, s); break;
        default: throw Error(ASPHER_EINVAL, "grid_size must be a power of two in [16, 1024]");
    }
}

}  // namespace
}  // namespace asb

extern "C" int aspher_periodic_matvec_noalloc(int grid_size, double domain_size, double E_star,
                                              int dtype, const void* x_dev, void* y_dev,
                                              void* stream) {
    try {
        if (grid_size < 16 || grid_size > asb::kNoAllocMaxNs || (grid_size & (grid_size - 1)))
            throw asb::Error(ASPHER_EINVAL,
                             "aspher_periodic_matvec_noalloc: grid_size must be a power of two "
                             "in [16, 1024] (the static scratch holds a 1024 grid)");
        if (!(domain_size > 0.0) || !std::isfinite(domain_size))
            throw asb::Error(ASPHER_EINVAL, "domain_size must be positive");
        if (!(E_star > 0.0) || !std::isfinite(E_star))
            throw asb::Error(ASPHER_EINVAL, "E_star must be positive");
        if (!x_dev || !y_dev)
            throw asb::Error(ASPHER_EINVAL, "aspher_periodic_matvec_noalloc: NULL buffer");
        if (((uintptr_t)x_dev | (uintptr_t)y_dev) % 16)
            throw asb::Error(ASPHER_EINVAL,
                             "aspher_periodic_matvec_noalloc: buffers must be 16-byte aligned");
        if (dtype != ASPHER_F64 && dtype != ASPHER_F32)
            throw asb::Error(ASPHER_EINVAL, "aspher_periodic_matvec_noalloc: dtype must be F32 or F64");
        cudaStream_t s = static_cast<cudaStream_t>(stream);
        asb::NaDevice& d = asb::na_setup(s);
        // same symbol scale as PeriodicFFTOperator (periodic_fft_operator.cpp:11-24)
        const double scale =
            domain_size / (M_PI * E_star * (double)grid_size * (double)grid_size);
        if (dtype == ASPHER_F64)
            asb::na_dispatch<double>(grid_size, d, scale, (const double*)x_dev, (double*)y_dev, s);
        else
            asb::na_dispatch<float>(grid_size, d, scale, (const float*)x_dev, (float*)y_dev, s);
        return ASPHER_OK;
    } catch (const asb::Error& e) {
        asb::set_last_error(e.what());
        return e.code;
    } catch (const std::exception& e) {
        asb::set_last_error(e.what());
        return ASPHER_ECUDA;
    }
}
