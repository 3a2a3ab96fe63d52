// Free-space (zero-padded Love/Boussinesq) and doubly periodic operators.
//
// Free space (reference: src/fft_operator.cpp:18-138): u = T (*) p, the
// aperiodic convolution with the Love table, evaluated on the (2Ns)^2
// padded grid.  Per apply:
//   row_fwd<LR=Ns, PAD>  : x rows (Ns reals, zero-padded to 2Ns) -> Ns+1 cols
//   col<LC=2Ns, PAD>     : pruned fwd FFT (upper half zero) * Kh, inverse
//                          FFT keeping rows [0, Ns)
//   row_inv<LR=Ns, PAD>  : c2r of length 2Ns keeping [0, Ns) -> y
// Kh is built on the device in FP64 (Love table -> embedded 2-D r2c via two
// real-row passes through a transposed buffer -> realness check), stored as
// real, even-folded in ky (rows [0, Ns]) and tiled for the column kernel.
//
// Periodic (reference: src/periodic_fft_operator.cpp:11-101): the symbol
// scale/|m| (scale = L/(pi E* Ns^2), m = (kx, signed ky), zero mode 0) is
// evaluated in FP64 inside the column kernel and cast to the working type.
#include "fft_kernels.cuh"
#include "fft_launch.cuh"
#include "functors.cuh"
#include "embed.cuh"
#include "kernel_tables.cuh"
#include "ops.hpp"
#include "pcg.hpp"
#include "reduce.cuh"

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace asb {

// ----------------------------------------------------------------------------
// twiddle tables
// ----------------------------------------------------------------------------
namespace {
void* g_tw[64][2] = {};  // [device][dbl]

void build_tw(int dev) {
    std::vector<double2> hd(2 * kMaxTw);
    std::vector<float2> hf(2 * kMaxTw);
    for (int L = 1; L <= kMaxTw; L <<= 1) {
        for (int k = 0; k < L; ++k) {
            const long double a = -2.0L * 3.14159265358979323846264338327950288L *
                                  (long double)k / (long double)L;
            const long double c = cosl(a), s = sinl(a);
            hd[L + k] = make_double2((double)c, (double)s);
            hf[L + k] = make_float2((float)c, (float)s);
        }
    }
    void *pd = nullptr, *pf = nullptr;
    ASB_CUDA(cudaMalloc(&pd, hd.size() * sizeof(double2)));
    ASB_CUDA(cudaMalloc(&pf, hf.size() * sizeof(float2)));
    ASB_CUDA(cudaMemcpy(pd, hd.data(), hd.size() * sizeof(double2), cudaMemcpyHostToDevice));
    ASB_CUDA(cudaMemcpy(pf, hf.data(), hf.size() * sizeof(float2), cudaMemcpyHostToDevice));
    g_tw[dev][1] = pd;
    g_tw[dev][0] = pf;
}
}  // namespace

const void* tw_table(bool dbl, int L) {
    int dev = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= 64) throw Error(-2, "device index out of range");
    if (!g_tw[dev][0]) {
        std::lock_guard<std::recursive_mutex> lk(setup_mutex());
        if (!g_tw[dev][0]) build_tw(dev);
    }
    if (L < 1 || L > kMaxTw) throw Error(-1, "twiddle length out of range");
    if (dbl) return static_cast<const double2*>(g_tw[dev][1]) + L;
    return static_cast<const float2*>(g_tw[dev][0]) + L;
}

bool is_pow2(long v) { return v > 0 && (v & (v - 1)) == 0; }

std::recursive_mutex& setup_mutex() {
    static std::recursive_mutex m;
    return m;
}

namespace {
std::atomic<long long> g_launches{0};
}
void count_launches(long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

void smem_optin(const void* func, int bytes) {
    if (bytes <= 48 * 1024) return;
    ASB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
}

// ----------------------------------------------------------------------------
// Love table (reference: src/boussinesq_kernel.cpp:44-106)
// ----------------------------------------------------------------------------
__global__ void love_table_kernel(double* __restrict__ tab, int Ns, double h, double scale) {
    const long n = (long)Ns * Ns;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int dy = (int)(i / Ns), dx = (int)(i % Ns);
        tab[i] = scale * love_uz_dev(dx * h, dy * h, 0.5 * h, 0.5 * h);
    }
}

// ----------------------------------------------------------------------------
// functors
// ----------------------------------------------------------------------------
// ---- Kh build functors (FP64) -------------------------------------------------
// Embedded table K(iy, ix) = T(|d(iy)|, |d(ix)|), d(i) = i (i < Ns) or i - M,
// with row/column Ns zero (fft_operator.cpp:31-44), generated on the fly.
struct LoadEmbedded {
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    const double* tab;
    int Ns, M;
    __device__ __forceinline__ double at(int iy, int ix) const {
        if (iy == Ns || ix == Ns) return 0.0;
        const int dy = iy < Ns ? iy : M - iy;
        const int dx = ix < Ns ? ix : M - ix;
        return tab[(size_t)dy * Ns + dx];
    }
    __device__ __forceinline__ double2 operator()(int row, int n) const {
        return make_double2(at(row, 2 * n), at(row, 2 * n + 1));
    }
};

// Pass A: Yt[k][row] = Re X (real by evenness in ix); tracks max|Im|, max|Re|.
// Pass B: canonical Kh[k * nk + row] = Re X / M^2 (ky = k, kx = row).
struct StoreRealTracked {
    double* out_t;  // pass A: transposed real, (Ns+1) x M
    int M;
    double* kh_d;   // pass B
    float* kh_f;
    int nk, ct_d, ct_f;
    double norm;
    unsigned long long* maxbits;  // [0] = max|Im|, [1] = max|Re| (as bit patterns)
    static constexpr bool kFinish = true;
    static constexpr bool kTiled = false;
    mutable double mi, mr;
    __device__ __forceinline__ void operator()(int row, int k, double2 X) const {
        if (out_t) {
            out_t[(size_t)k * M + row] = X.x;
        } else {
            kh_d[(size_t)k * nk + row] = X.x * norm;
        }
        mi = fmax(mi, fabs(X.y));
        mr = fmax(mr, fabs(X.x));
    }
    __device__ void finish(double* scratch) const {
        double v[2] = {mi, mr};
        const int kinds[2] = {2, 2};
        block_reduce<2>(v, kinds, scratch);
        if (threadIdx.x == 0) {
            atomicMax(&maxbits[0], (unsigned long long)__double_as_longlong(v[0]));
            atomicMax(&maxbits[1], (unsigned long long)__double_as_longlong(v[1]));
        }
    }
};

// The functors are passed by value; StoreRealTracked keeps per-thread maxima
// in mutable members initialised to zero by the host copy.

// Split form of the two Kh passes, for rows of M = 2 Ns reals whose complex
// FFT (length Ns) does not fit one CTA (FP64 at Ns > 8192): the real DFT of
// a row is assembled from the real DFTs of its even and odd samples,
//   X[k] = E[k] + w_M^k O[k],  k in [0, Ns],  w_M = exp(-2 pi i / M),
// with E[Ns - k] = conj E[k] (and O likewise) for the upper half.  The first
// pass stores E (row_fwd of the even samples, StoreCplxRows), the second
// transforms the odd samples and combines while storing (StoreSplitCombine).
struct LoadEmbeddedPar {  // z[n] = (x[4n + p], x[4n + 2 + p]) of an embedded row
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    LoadEmbedded e;
    int p;
    __device__ __forceinline__ double2 operator()(int row, int n) const {
        return make_double2(e.at(row, 4 * n + p), e.at(row, 4 * n + 2 + p));
    }
};
struct LoadRealRowsPar {  // the same sampling of plain rows
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    const double* x;
    int pitch, p;
    __device__ __forceinline__ double2 operator()(int row, int n) const {
        const double* r = x + (size_t)row * pitch;
        return make_double2(r[4 * n + p], r[4 * n + 2 + p]);
    }
};
struct StoreCplxRows {
    static constexpr bool kFinish = false;
    static constexpr bool kTiled = false;
    double2* out;
    int pitch;
    __device__ __forceinline__ void operator()(int row, int k, double2 X) const {
        out[(size_t)row * pitch + k] = X;
    }
    __device__ void finish(double*) const {}
};
struct StoreSplitCombine {
    static constexpr bool kFinish = true;
    static constexpr bool kTiled = false;
    const double2* E;     // even-sample half spectra, pitch entries per row
    int pitch;
    const double2* twm;   // exp(-2 pi i k / M), k < M
    int half;             // M / 2 = Ns
    StoreRealTracked inner;
    __device__ __forceinline__ void operator()(int row, int k, double2 O) const {
        const double2 e = E[(size_t)row * pitch + k];
        inner(row, k, cadd(e, cmul(O, __ldg(&twm[k]))));
        const int k2 = half - k;
        inner(row, k2, cadd(cconj(e), cmul(cconj(O), __ldg(&twm[k2]))));
    }
    __device__ void finish(double* scratch) const { inner.finish(scratch); }
};

// ----------------------------------------------------------------------------
// launch-variant selection: a default per (backend, precision, Ns), overridden
// process-wide by the autotuner (Operator::autotune) or set per operator
// ----------------------------------------------------------------------------
namespace {
std::mutex g_tuned_mu;
std::map<std::tuple<int, int, int>, std::pair<int, int>> g_tuned;
}  // namespace

// Fastest (row, column) variant pairs measured on B200: every pair set on
// one operator (aspher_op_set_variants) and its apply timed with CUDA
// events, L2 flushed between applies, median of 15; sizes not listed use
// variant 0.  Operator::autotune repeats the search in-process.
void default_variants(int kind, int dbl, int Ns, int& rv, int& cv) {
    static const int table[][5] = {
        // kind, dbl, Ns, row variant, column variant
        {0, 0, 256, 2, 3}, {0, 0, 512, 2, 1}, {0, 0, 1024, 1, 1}, {0, 0, 2048, 1, 0},
        {0, 0, 4096, 0, 1}, {0, 0, 8192, 1, 2}, {0, 1, 256, 1, 1}, {0, 1, 512, 1, 1},
        {0, 1, 1024, 0, 1}, {0, 1, 2048, 2, 0}, {0, 1, 4096, 0, 0}, {1, 0, 256, 3, 3},
        {1, 0, 512, 0, 3}, {1, 0, 1024, 2, 3}, {1, 0, 2048, 1, 1}, {1, 0, 4096, 1, 0},
        {1, 0, 8192, 0, 1}, {1, 1, 256, 3, 3}, {1, 1, 512, 1, 3}, {1, 1, 1024, 2, 2},
        {1, 1, 2048, 2, 0}, {1, 1, 4096, 2, 0}, {1, 1, 8192, 0, 0},
    };
    rv = 0;
    cv = 0;
    for (const auto& e : table)
        if (e[0] == kind && e[1] == dbl && e[2] == Ns) {
            rv = e[3];
            cv = e[4];
            return;
        }
}

void tuned_variants(int kind, int dbl, int Ns, int& rv, int& cv) {
    {
        std::lock_guard<std::mutex> lk(g_tuned_mu);
        auto it = g_tuned.find(std::make_tuple(kind, dbl, Ns));
        if (it != g_tuned.end()) {
            rv = it->second.first;
            cv = it->second.second;
            return;
        }
    }
    default_variants(kind, dbl, Ns, rv, cv);
}

void record_tuned(int kind, int dbl, int Ns, int rv, int cv) {
    std::lock_guard<std::mutex> lk(g_tuned_mu);
    g_tuned[std::make_tuple(kind, dbl, Ns)] = std::make_pair(rv, cv);
}

// ----------------------------------------------------------------------------
// launch attributes and persistent grids (the launchers are in fft_launch.cuh)
// ----------------------------------------------------------------------------
namespace {
std::mutex g_attr_mu;
std::map<std::pair<const void*, int>, int> g_attr_done;
}  // namespace

// Max dynamic shared memory and the shared-memory carveout, once per kernel
// per device.  The carveout asks for the shared memory of as many CTAs as
// fit on an SM (registers, threads and shared memory counted with every
// byte available to shared memory) and no more: the rest of the SM's
// unified L1 / shared storage stays L1 cache, which holds the twiddle
// tables and multiplier rows the pass kernels read through the read-only
// path.  The driver rounds the request up to a supported split.
void fft_attrs(const void* func, int bytes) {
    int dev = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(g_attr_mu);
    auto key = std::make_pair(func, dev);
    auto it = g_attr_done.find(key);
    if (it != g_attr_done.end() && it->second >= bytes) return;
    if (bytes > 48 * 1024)
        ASB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes));
    ASB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout,
                                  cudaSharedmemCarveoutMaxShared));
    cudaFuncAttributes fa{};
    ASB_CUDA(cudaFuncGetAttributes(&fa, func));
    int per_sm = 0, sm_bytes = 0, reserved = 0;
    ASB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, fa.maxThreadsPerBlock,
                                                           bytes));
    ASB_CUDA(cudaDeviceGetAttribute(&sm_bytes, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev));
    ASB_CUDA(cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev));
    if (per_sm > 0 && sm_bytes > 0) {
        const long need = (long)per_sm * ((long)bytes + (long)fa.sharedSizeBytes + reserved);
        const int pct = (int)std::min<long>(100, (need * 100 + sm_bytes - 1) / sm_bytes);
        ASB_CUDA(cudaFuncSetAttribute(func, cudaFuncAttributePreferredSharedMemoryCarveout, pct));
    }
    g_attr_done[key] = bytes;
}

// Persistent grid of a pass kernel: at most as many CTAs as fit on the device
// at once (occupancy x SMs, cached per kernel, block shape and device), and
// no more than the units (row groups / column tiles) to process.
namespace {
std::mutex g_occ_mu;
std::map<std::tuple<const void*, int, int, int>, int> g_occ;
}  // namespace
int persistent_blocks(const void* func, int threads, int smem, int units) {
    int dev = 0;
    ASB_CUDA(cudaGetDevice(&dev));
    const auto key = std::make_tuple(func, threads, smem, dev);
    int resident = 0;
    {
        std::lock_guard<std::mutex> lk(g_occ_mu);
        auto it = g_occ.find(key);
        if (it != g_occ.end()) resident = it->second;
    }
    if (!resident) {
        int per_sm = 0, nsm = 0;
        ASB_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, func, threads, smem));
        ASB_CUDA(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        resident = (per_sm > 0 ? per_sm : 1) * nsm;
        std::lock_guard<std::mutex> lk(g_occ_mu);
        g_occ[key] = resident;
    }
    return units < resident ? units : resident;
}

// the two launches of the split column transform (variant 0 only): parity 0
// writes its half to acc, parity 1 adds it and writes the column in place
template <typename T, int LH, int NCM1, class Mult>
void launch_col_split(cplx<T>* spec, cplx<T>* acc, int nrows, Mult m, cudaStream_t s,
                      const int* gate, int B = 1) {
    constexpr int V = vclamp(LH, 0);
    constexpr int ct = col_ct_v<T>(LH, NCM1, V), thr = col_threads<T>(LH, NCM1, V);
    constexpr int sm = col_smem<T>(LH, ct);
    auto k0 = col_split_kernel<T, LH, NCM1, V, 0, Mult>;
    auto k1 = col_split_kernel<T, LH, NCM1, V, 1, Mult>;
    fft_attrs((const void*)k0, sm);
    fft_attrs((const void*)k1, sm);
    const dim3 grid(NCM1 / ct + 1, B);
    k0<<<grid, thr, sm, s>>>(spec, acc, nrows, m, tw<T>(LH), tw<T>(2 * LH), gate);
    k1<<<grid, thr, sm, s>>>(spec, acc, nrows, m, tw<T>(LH), tw<T>(2 * LH), gate);
}

#define ASB_V_SWITCH(VV, L, ...)                                                   \
    switch (VV) {                                                                  \
        case 0: { constexpr int V = vclamp(L, 0); __VA_ARGS__; } break;            \
        case 1: { constexpr int V = vclamp(L, 1); __VA_ARGS__; } break;            \
        case 2: { constexpr int V = vclamp(L, 2); __VA_ARGS__; } break;            \
        case 3: { constexpr int V = vclamp(L, 3); __VA_ARGS__; } break;            \
        default: throw Error(-1, "FFT launch variant out of range");              \
    }

// ALLV = false: launch variant 0 whatever v is (one instantiation per pass;
// the grids above kMaxVariantNs)
template <typename T, int LR, bool PAD, bool ALLV = true, class Load, class Store>
void row_fwd_v(int v, Load ld, Store st, int nrows, cudaStream_t s, const int* gate, int B) {
    if constexpr (!ALLV) {
        launch_row_fwd<T, LR, PAD, vclamp(LR, 0), Load, Store>(ld, st, nrows, s, gate, B);
    } else {
        ASB_V_SWITCH(v, LR, (launch_row_fwd<T, LR, PAD, V, Load, Store>(ld, st, nrows, s, gate, B)));
    }
}
template <typename T, int LR, bool PAD, bool ALLV = true, class Load, class Store>
void row_inv_v(int v, Load ld, Store st, int nrows, cudaStream_t s, const int* gate, int B) {
    if constexpr (!ALLV) {
        launch_row_inv<T, LR, PAD, vclamp(LR, 0), Load, Store>(ld, st, nrows, s, gate, B);
    } else {
        ASB_V_SWITCH(v, LR, (launch_row_inv<T, LR, PAD, V, Load, Store>(ld, st, nrows, s, gate, B)));
    }
}
template <typename T, int LC, int NCM1, bool PAD, bool ALLV = true, class Mult>
void col_v(int v, cplx<T>* spec, int nrows, Mult m, cudaStream_t s, const int* gate, int B) {
    if constexpr (!ALLV) {
        launch_col<T, LC, NCM1, PAD, vclamp(LC, 0), Mult>(spec, nrows, m, s, gate, B);
    } else {
        ASB_V_SWITCH(v, LC, (launch_col<T, LC, NCM1, PAD, V, Mult>(spec, nrows, m, s, gate, B)));
    }
}
// tile width of column variant v (runtime view of the constexpr table)
template <typename T, int LC, int NCM1>
int col_ct_rt(int v) {
    int ct = 1;
    ASB_V_SWITCH(v, LC, ct = col_ct_v<T>(LC, NCM1, V));
    return ct;
}

// ----------------------------------------------------------------------------
// per-size implementation
// ----------------------------------------------------------------------------
template <typename T, int NS>
struct FreeImpl {
    static constexpr int LR = NS, LC = 2 * NS;
    // the length-2Ns column in one CTA's shared memory (all sizes but FP64
    // at Ns = 8192); otherwise the column pass runs as two length-Ns halves
    // (col_split_kernel), instantiated for Ns >= kSplitMin
    static constexpr bool kFits = col_fits<T>(LC);
    static constexpr bool kSplitOK = NS >= kSplitMin && col_fits<T>(LR);
    // rows and columns in one CTA each (every size but FP64 above 8192)
    static constexpr bool kSupported = row_smem_v<T>(LR, 0) <= kSmemPerSM && (kFits || kSplitOK);
    static constexpr bool kAllV = NS <= kMaxVariantNs;
    static bool split(const Operator& op) { return !kFits || (kSplitOK && op.split_cols); }
    // spectrum sized for the widest tile (16 columns); the split form keeps
    // its first half-column result in a second spectrum-shaped block after
    // the B instances' spectra
    static size_t spec_elems(bool sp) { return (size_t)(LR + 16) * NS * (sp ? 2 : 1); }
    static int ct(int cv, bool sp) {
        if (sp) return col_ct_v<T>(LR, LR, vclamp(LR, 0));
        return kAllV ? col_ct_rt<T, LC, LR>(cv) : col_ct_v<T>(LC, LR, vclamp(LC, 0));
    }

    // row_fwd(ld) -> col(x Kh) -> row_inv(st); ld / st see the Ns x Ns field(s)
    template <class Load, class Store>
    static void apply(const Operator& op, Load ld, Store st, cplx<T>* spec, cudaStream_t s,
                      const int* gate, int B, const T* kh_over = nullptr) {
        if constexpr (!kSupported) {
            throw Error(-1, "free-space FP64 apply above grid_size 8192 is not supported (its "
                            "rows and half columns do not fit one CTA's shared memory); use FP32");
        } else {
            const int dbl = sizeof(T) == 8;
            const int rv = op.rowv[dbl], cv = op.colv[dbl], c = op.ct[dbl];
            const T* kh = kh_over ? kh_over : (dbl ? (const T*)op.kh_d : (const T*)op.kh_f);
            const long bsp = (long)(LR / c + 1) * NS * c;
            row_fwd_v<T, LR, true, kAllV>(rv, ld, StoreTiled<T>{spec, NS, c, bsp}, NS, s, gate, B);
            if (split(op)) {
                if constexpr (kSplitOK)
                    launch_col_split<T, LR, LR>(spec, spec + (size_t)B * bsp, NS,
                                                KhMult<T>{kh, NS + 1, LC, c}, s, gate, B);
            } else {
                if constexpr (kFits)
                    col_v<T, LC, LR, true, kAllV>(cv, spec, NS, KhMult<T>{kh, NS + 1, LC, c}, s,
                                                  gate, B);
            }
            row_inv_v<T, LR, true, kAllV>(rv, LoadTiled<T>{spec, NS, c, bsp}, st, NS, s, gate, B);
            count_launches(split(op) ? 4 : 3);
            ASB_CUDA(cudaGetLastError());
        }
    }

    static void matvec(const Operator& op, const T* x, T* y, cplx<T>* spec, cudaStream_t s,
                       const int* gate, int B, const PkState* sc) {
        const long bx = (long)NS * NS;
        apply(op, LoadRealRows<T>{x, NS, bx, sc}, StoreRealRows<T>{y, NS, bx}, spec, s, gate, B);
    }
};

template <typename T, int NS>
struct PeriodicImpl {
    static constexpr int LR = NS / 2, LC = NS;
    // rows and columns in one CTA each (every size but FP64 above 8192)
    static constexpr bool kSupported = row_smem_v<T>(LR, 0) <= kSmemPerSM && col_fits<T>(LC);
    static constexpr bool kAllV = NS <= kMaxVariantNs;
    static size_t spec_elems() { return (size_t)(LR + 16) * NS; }
    static int ct(int cv) {
        return kAllV ? col_ct_rt<T, LC, LR>(cv) : col_ct_v<T>(LC, LR, vclamp(LC, 0));
    }

    template <class Load, class Mult, class Store>
    static void apply(int rv, int cv, Load ld, Mult mult, Store st, cplx<T>* spec, cudaStream_t s,
                      const int* gate, int B) {
        if constexpr (!kSupported) {
            throw Error(-1, "periodic FP64 apply above grid_size 8192 is not supported (its "
                            "column does not fit one CTA's shared memory); use FP32");
        } else {
            const int c = ct(cv);
            const long bsp = (long)(LR / c + 1) * NS * c;
            row_fwd_v<T, LR, false, kAllV>(rv, ld, StoreTiled<T>{spec, NS, c, bsp}, NS, s, gate, B);
            col_v<T, LC, LR, false, kAllV>(cv, spec, NS, mult, s, gate, B);
            row_inv_v<T, LR, false, kAllV>(rv, LoadTiled<T>{spec, NS, c, bsp}, st, NS, s, gate, B);
            count_launches(3);
            ASB_CUDA(cudaGetLastError());
        }
    }

    // the multiplier scale / |m| from the operator's table of this precision
    // (the values PeriodicMult forms per element, one load instead of an
    // FP64 square root and division)
    static KhMult<T> mult(const Operator& op) {
        const int dbl = sizeof(T) == 8;
        const T* tab = dbl ? (const T*)(const void*)op.psym_d : (const T*)(const void*)op.psym_f;
        return KhMult<T>{tab, NS / 2 + 1, NS, op.ct[dbl]};
    }

    static void matvec(const Operator& op, const T* x, T* y, cplx<T>* spec, cudaStream_t s,
                       const int* gate, int B, const PkState* sc) {
        const int dbl = sizeof(T) == 8;
        const long bx = (long)NS * NS;
        apply(op.rowv[dbl], op.colv[dbl], LoadRealRows<T>{x, NS, bx, sc}, mult(op),
              StoreRealRows<T>{y, NS, bx}, spec, s, gate, B);
    }
};

// ----------------------------------------------------------------------------
// full-grid |k| preconditioner (reference: src/fourier_precond.cpp:12-116)
// ----------------------------------------------------------------------------
template <typename T>
struct LoadMaskCentered {  // contact ? g - T(gsum/ng) : 0, pairwise; g = v - T(alpha)
    static constexpr bool kTiled = false;
    static constexpr bool kRaw = false;
    const T* g;
    const uint8_t* mask;
    const PkState* st;
    int pitch;
    long bs;  // batch stride (elements); instance blockIdx.y uses st[blockIdx.y]
    __device__ __forceinline__ cplx<T> operator()(int row, int n) const {
        const PkState* sb = st + blockIdx.y;
        const int nc = sb->nc;
        const T gm = nc ? (T)(sb->gcs / nc) : T(0);
        // the solve loop keeps g uncentred (centred by Real(alpha) on the fly;
        // alpha is 0 for the standalone preconditioner)
        const T aT = (T)sb->alpha;
        const size_t i = blockIdx.y * bs + (size_t)row * pitch + 2 * n;
        const cplx<T> v = *reinterpret_cast<const cplx<T>*>(g + i);
        const uchar2 m = *reinterpret_cast<const uchar2*>(mask + i);
        return mk<T>(m.x ? (T)((T)(v.x - aT) - gm) : T(0), m.y ? (T)((T)(v.y - aT) - gm) : T(0));
    }
};

template <typename T>
struct FourierMult {  // |k| / Ns^2 as the reference's float table, cast to T
    int Ns;
    float norm;
    __device__ __forceinline__ cplx<T> operator()(cplx<T> X, int kx, int ky) const {
        const int kof = ky < Ns / 2 ? ky : ky - Ns;
        const float w = (kx == 0 && ky == 0) ? 0.0f : norm * hypotf((float)kx, (float)kof);
        return cscale(X, (T)w);
    }
};

template <typename T>
struct StoreGather {  // z = contact ? G : 0; contact sum of G -> zmean
    static constexpr bool kTiled = false;
    T* z;
    const uint8_t* mask;
    int pitch;
    PkState* st;
    double* part;
    long bs;  // batch stride (elements); instance blockIdx.y uses st / part of its own
    static constexpr bool kFinish = true;
    double zs;
    __device__ __forceinline__ void operator()(int row, int n, cplx<T> v) {
        const size_t i = blockIdx.y * bs + (size_t)row * pitch + 2 * n;
        const uchar2 m = *reinterpret_cast<const uchar2*>(mask + i);
        *reinterpret_cast<cplx<T>*>(z + i) = mk<T>(m.x ? v.x : T(0), m.y ? v.y : T(0));
        if (m.x) zs += (double)v.x;
        if (m.y) zs += (double)v.y;
    }
    __device__ void finish(double*) {
        double a[1] = {zs};
        const int kinds[1] = {0};
        PkState* sb = st + blockIdx.y;
        double* pb = part + (size_t)blockIdx.y * kPartStride;
        if (grid_reduce_last<1>(a, kinds, pb, &sb->counter[11]) && threadIdx.x == 0) {
            const int nc = sb->nc;
            sb->zmean = nc ? (double)(T)(a[0] / nc) : 0.0;
            sb->pc++;
        }
    }
};

template <typename T, int NS>
struct FourierImpl {
    using PI = PeriodicImpl<T, NS>;
    static void run(Operator& op, const T* g, const uint8_t* mask, PkState* st, T* z,
                    double* part, cudaStream_t s, const int* gate, int B, void* spec_b) {
        cplx<T>* spec = static_cast<cplx<T>*>(spec_b ? spec_b : op.spectrum(sizeof(T) == 8, s));
        int rv = 0, cv = 0;
        tuned_variants(OP_PERIODIC, sizeof(T) == 8, NS, rv, cv);
        const float norm = 1.0f / ((float)NS * (float)NS);
        const long bx = (long)NS * NS;
        PI::apply(rv, cv, LoadMaskCentered<T>{g, mask, st, NS, bx}, FourierMult<T>{NS, norm},
                  StoreGather<T>{z, mask, NS, st, part, bx, 0.0}, spec, s, gate, B);
    }
};

// Kh build for the free-space operator of size NS (FP64): canonical real
// spectrum kh_canon[ky * (Ns+1) + kx], ky, kx in [0, Ns].
template <int NS>
struct KhBuild {
    // the split form (see StoreSplitCombine) where the FP64 row does not fit
    // one CTA, or where the operator's creation flags ask for it
    // (cross-checks), for Ns >= kSplitMin
    static constexpr bool kRowFits = row_smem_v<double>(NS, 0) <= kSmemPerSM;
    static bool split(const Operator& op) {
        if (!kRowFits) return true;
        return NS >= kSplitMin && op.split_kh;
    }
    static void run(Operator& op) {
        const size_t nk = (size_t)(NS + 1) * (NS + 1);
        ASB_CUDA(cudaMalloc(&op.kh_canon, nk * sizeof(double)));
        op.max_im_ratio = build(op, op.table, op.kh_canon);
    }
    // the canonical spectrum of an even table (tab, Ns x Ns) into canon
    // ((Ns+1)^2); returns the realness ratio, throws when it fails
    static double build(const Operator& op, const double* table, double* canon) {
        constexpr int LR = NS, M = 2 * NS;
        double* yt = nullptr;
        unsigned long long* mx = nullptr;
        ASB_CUDA(cudaMalloc(&yt, (size_t)(NS + 1) * M * sizeof(double)));
        ASB_CUDA(cudaMalloc(&mx, 4 * sizeof(unsigned long long)));
        ASB_CUDA(cudaMemset(mx, 0, 4 * sizeof(unsigned long long)));
        StoreRealTracked sa{yt, M, nullptr, nullptr, 0, 0, 0, 0.0, mx, 0.0, 0.0};
        StoreRealTracked sb{nullptr, M, canon, nullptr, NS + 1, 0, 0,
                            1.0 / ((double)M * (double)M), mx + 2, 0.0, 0.0};
        const LoadEmbedded emb{table, NS, M};
        if (split(op)) {
            if constexpr (NS >= kSplitMin) {
                constexpr int LH = NS / 2;  // real length Ns per parity
                double2* E = nullptr;
                ASB_CUDA(cudaMalloc(&E, (size_t)M * (LH + 1) * sizeof(double2)));
                const double2* twm = tw<double>(M);
                // pass A over the M rows of the embedded table
                launch_row_fwd<double, LH, false, 0>(LoadEmbeddedPar{emb, 0},
                                                     StoreCplxRows{E, LH + 1}, M, nullptr, nullptr);
                launch_row_fwd<double, LH, false, 0>(
                    LoadEmbeddedPar{emb, 1}, StoreSplitCombine{E, LH + 1, twm, NS, sa}, M, nullptr,
                    nullptr);
                ASB_CUDA(cudaGetLastError());
                // pass B over the Ns+1 rows of the transposed buffer
                launch_row_fwd<double, LH, false, 0>(LoadRealRowsPar{yt, M, 0},
                                                     StoreCplxRows{E, LH + 1}, NS + 1, nullptr,
                                                     nullptr);
                launch_row_fwd<double, LH, false, 0>(
                    LoadRealRowsPar{yt, M, 1}, StoreSplitCombine{E, LH + 1, twm, NS, sb}, NS + 1,
                    nullptr, nullptr);
                ASB_CUDA(cudaGetLastError());
                ASB_CUDA(cudaDeviceSynchronize());
                ASB_CUDA(cudaFree(E));
            }
        } else {
            if constexpr (kRowFits) {
                // pass A over the M rows of the embedded table (real by evenness in ix)
                launch_row_fwd<double, LR, false, 0>(emb, sa, M, nullptr, nullptr);
                ASB_CUDA(cudaGetLastError());
                // pass B over the Ns+1 rows of the transposed buffer (each M long)
                launch_row_fwd<double, LR, false, 0>(LoadRealRows<double>{yt, M, 0}, sb, NS + 1,
                                                     nullptr, nullptr);
                ASB_CUDA(cudaGetLastError());
            }
        }
        unsigned long long h[4];
        ASB_CUDA(cudaMemcpy(h, mx, sizeof(h), cudaMemcpyDeviceToHost));
        ASB_CUDA(cudaFree(yt));
        ASB_CUDA(cudaFree(mx));
        double v[4];
        for (int i = 0; i < 4; ++i) std::memcpy(&v[i], &h[i], sizeof(double));
        const double ra = v[1] > 0 ? v[0] / v[1] : 0.0;
        const double rbt = v[3] > 0 ? v[2] / v[3] : 0.0;
        const double ratio = ra > rbt ? ra : rbt;
        // fft_operator.cpp:57-60: the embedding is even, so the spectrum is real
        if (v[0] > 1e-10 * v[1] || v[2] > 1e-10 * v[3])
            throw Error(-3, "FFTOperator: kernel spectrum has a non-negligible imaginary "
                            "part; wrap-around embedding is broken");
        return ratio;
    }
};

// ----------------------------------------------------------------------------
// Real-space kernel of the periodic operator on an Nl torus (embedded
// periodic operators).  The reference applies c2r(sigma r2c(x)) with
// sigma(kx, ky) = scale / |m| (0 at the zero mode; periodic_fft_operator.cpp:
// 31-45); with sigma even in each wavenumber that is the circulant
//   y(i) = sum_j T((i - j) mod Nl) x(j),
//   T(dy, dx) = sum_{ky, kx < Nl} sigma cos(2 pi kx dx / Nl) cos(2 pi ky dy / Nl),
// which the free-space pipeline computes as the padded linear convolution of
// the block with T over offsets |d| < Nl (T even: T(-d) = T(Nl - d) = T(d)).
// T is formed as two cosine sums over the half range of each wavenumber
// (weights 2 but at 0 and the even-Nl Nyquist index), each accumulated with
// Kahan compensation in FP64, so every entry carries a few roundings of the
// largest term (T(0, 0) ~ scale Nl) rather than sqrt(Nl) of them.
// ----------------------------------------------------------------------------
__global__ void k_cos_table(int Nl, double* __restrict__ c) {
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < Nl; r += gridDim.x * blockDim.x)
        c[r] = cospi(2.0 * (double)r / (double)Nl);
}

__device__ __forceinline__ double half_weight(int k, int Nl) {
    return (k == 0 || 2 * k == Nl) ? 1.0 : 2.0;
}

__device__ __forceinline__ void kahan_add(double& sum, double& comp, double term) {
    const double y = term - comp;
    const double t = sum + y;
    comp = (t - sum) - y;
    sum = t;
}

// A[ky][dx] = sum_{kx < nh} w(kx) sigma(kx, ky) cos(2 pi kx dx / Nl), ky < nh
// (block: one ky, threads over dx; shared: the cosine table and sigma's row)
// symbol 0: scale / |m| (the periodic operator); 1: the full-grid |k|
// preconditioner's float symbol, float(normf |k|) with normf = float(1 / Nl^2)
// as the reference stores it (fourier_precond.cpp:12-28); both 0 at DC
__global__ void k_periodic_rows(int Nl, int symbol, double scale, const double* __restrict__ ctab,
                                double* __restrict__ A) {
    extern __shared__ double sh[];
    const int nh = Nl / 2 + 1;
    double* cs = sh;        // Nl cosines
    double* sg = sh + Nl;   // nh weighted symbol values of this ky
    const int ky = blockIdx.y;
    for (int r = threadIdx.x; r < Nl; r += blockDim.x) cs[r] = ctab[r];
    for (int kx = threadIdx.x; kx < nh; kx += blockDim.x) {
        const double m2 = (double)kx * kx + (double)ky * ky;
        double sym = 0.0;
        if (m2 > 0.0) {
            if (symbol == 0) {
                sym = scale / sqrt(m2);
            } else {
                const float normf = 1.0f / ((float)Nl * (float)Nl);
                sym = (double)(normf * hypotf((float)kx, (float)ky));
            }
        }
        sg[kx] = half_weight(kx, Nl) * sym;
    }
    __syncthreads();
    const int dx = blockIdx.x * blockDim.x + threadIdx.x;
    if (dx >= Nl) return;
    double sum = 0.0, comp = 0.0;
    int idx = 0;  // (dx kx) mod Nl
    for (int kx = 0; kx < nh; ++kx) {
        kahan_add(sum, comp, sg[kx] * cs[idx]);
        idx += dx;
        if (idx >= Nl) idx -= Nl;
    }
    A[(size_t)ky * Nl + dx] = sum;
}

// T[dy][dx] = sum_{ky < nh} w(ky) cos(2 pi ky dy / Nl) A[ky][dx], written
// into the Ns x Ns table (pitch Ns) whose entries at |d| >= Nl stay zero
__global__ void k_periodic_cols(int Nl, int Ns, const double* __restrict__ ctab,
                                const double* __restrict__ A, double* __restrict__ tab) {
    const int nh = Nl / 2 + 1;
    const int dy = blockIdx.y;
    const int dx = blockIdx.x * blockDim.x + threadIdx.x;
    if (dx >= Nl) return;
    double sum = 0.0, comp = 0.0;
    int idx = 0;  // (dy ky) mod Nl
    for (int ky = 0; ky < nh; ++ky) {
        kahan_add(sum, comp, half_weight(ky, Nl) * __ldg(&ctab[idx]) * A[(size_t)ky * Nl + dx]);
        idx += dy;
        if (idx >= Nl) idx -= Nl;
    }
    tab[(size_t)dy * Ns + dx] = sum;
}

void periodic_kernel_table(int Nl, int Ns, double scale, double* tab, int symbol = 0) {
    const int nh = Nl / 2 + 1;
    double *ctab = nullptr, *A = nullptr;
    ASB_CUDA(cudaMalloc(&ctab, (size_t)Nl * sizeof(double)));
    ASB_CUDA(cudaMalloc(&A, (size_t)nh * Nl * sizeof(double)));
    ASB_CUDA(cudaMemset(tab, 0, (size_t)Ns * Ns * sizeof(double)));
    k_cos_table<<<(Nl + 255) / 256, 256>>>(Nl, ctab);
    const int smem = (Nl + nh) * (int)sizeof(double);
    smem_optin((const void*)k_periodic_rows, smem);
    k_periodic_rows<<<dim3((Nl + 127) / 128, nh), 128, smem>>>(Nl, symbol, scale, ctab, A);
    k_periodic_cols<<<dim3((Nl + 127) / 128, Nl), 128>>>(Nl, Ns, ctab, A, tab);
    count_launches(3);
    ASB_CUDA(cudaGetLastError());
    ASB_CUDA(cudaDeviceSynchronize());
    cudaFree(ctab);
    cudaFree(A);
}

// tiled copy of the canonical Kh for column tile width ct (both precisions)
__global__ void k_retile_kh(int Ns, const double* __restrict__ canon, int ct_d,
                            double* __restrict__ kd, int ct_f, float* __restrict__ kf) {
    const int nk = Ns + 1;
    const long n = (long)nk * nk;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int ky = (int)(i / nk), kx = (int)(i % nk);
        const double v = canon[i];
        if (kd) kd[(size_t)(kx / ct_d) * nk * ct_d + (size_t)ky * ct_d + (kx % ct_d)] = v;
        if (kf) kf[(size_t)(kx / ct_f) * nk * ct_f + (size_t)ky * ct_f + (kx % ct_f)] = (float)v;
    }
}

// The periodic multiplier (periodic_fft_operator.cpp:34-47) as a table:
// w(kx, kf) = scale / sqrt(kx^2 + kf^2) in FP64 (0 at the mean), the value
// PeriodicMult forms per element, for kx in [0, ncols) (columns past Ns/2
// pad the last tile: 0) and kf = |m_y| in [0, Ns/2], tiled for column tile
// width ct as Kh is: [kx / ct][kf][kx % ct]
__global__ void k_periodic_symbol(int Ns, double scale, int ncols, int ct,
                                  double* __restrict__ sd, float* __restrict__ sf) {
    const int nk = Ns / 2 + 1;
    const long n = (long)ncols * nk;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n;
         i += (long)gridDim.x * blockDim.x) {
        const int kf = (int)(i / ncols), kx = (int)(i % ncols);
        const double m2 = (double)kx * kx + (double)kf * kf;
        const double w = (kx <= Ns / 2 && m2 > 0.0) ? scale / sqrt(m2) : 0.0;
        const size_t at = (size_t)(kx / ct) * nk * ct + (size_t)kf * ct + (kx % ct);
        if (sd) sd[at] = w;
        if (sf) sf[at] = (float)w;
    }
}

// ----------------------------------------------------------------------------
// size dispatch
// ----------------------------------------------------------------------------
#define ASB_SIZE_SWITCH(NSV, ...)                      \
    switch (NSV) {                                      \
        case 16: { constexpr int NS = 16; __VA_ARGS__; } break;     \
        case 32: { constexpr int NS = 32; __VA_ARGS__; } break;     \
        case 64: { constexpr int NS = 64; __VA_ARGS__; } break;     \
        case 128: { constexpr int NS = 128; __VA_ARGS__; } break;   \
        case 256: { constexpr int NS = 256; __VA_ARGS__; } break;   \
        case 512: { constexpr int NS = 512; __VA_ARGS__; } break;   \
        case 1024: { constexpr int NS = 1024; __VA_ARGS__; } break; \
        case 2048: { constexpr int NS = 2048; __VA_ARGS__; } break; \
        case 4096: { constexpr int NS = 4096; __VA_ARGS__; } break; \
        case 8192: { constexpr int NS = 8192; __VA_ARGS__; } break; \
        case 16384: { constexpr int NS = 16384; __VA_ARGS__; } break; \
        default: throw Error(-1, "grid_size must be a power of two in [16, 16384]"); \
    }

Operator::Operator(int kind_, int Ns_, double L_, double E_, int flags)
    : kind(kind_), Ns(Ns_), L(L_), E_star(E_), Nl(Ns_), backend(kind_) {
    if (kind != OP_FFT && kind != OP_PERIODIC) throw Error(-1, "unknown operator kind");
    if (Nl < 2 || Nl > kMaxNs) throw Error(-1, "grid_size must be in [2, 16384]");
    if (!(L > 0.0) || !std::isfinite(L)) throw Error(-1, "domain_size must be positive");
    if (!(E_star > 0.0) || !std::isfinite(E_star)) throw Error(-1, "E_star must be positive");
    if (flags & ~(OPF_SPLIT_COLUMNS | OPF_SPLIT_KH)) throw Error(-1, "unknown operator flags");
    if (!is_pow2(Nl) || Nl < 16) {
        // embedded: the free-space pipeline of the next power of two
        if (flags) throw Error(-1, "operator flags need a power-of-two grid_size in [16, 16384]");
        int nc = 16;
        while (nc < Nl) nc *= 2;
        Ns = nc;
        kind = OP_FFT;
    }
    std::lock_guard<std::recursive_mutex> setup(setup_mutex());
    ASB_CUDA(cudaGetDevice(&device));
    (void)tw_table(false, 2);
    // cross-check forms: the free-space column pass in its split (two
    // half-length) form and the FP64 Kh build from even / odd row samples at
    // every size >= kSplitMin, the forms FP64 at Ns = 8192 and 16384 need
    split_cols = kind == OP_FFT && Ns >= kSplitMin && (flags & OPF_SPLIT_COLUMNS);
    split_kh = kind == OP_FFT && Ns >= kSplitMin && (flags & OPF_SPLIT_KH);
    if (backend == OP_PERIODIC) scale = L / (M_PI * E_star * (double)Nl * Nl);
    if (kind == OP_FFT) {
        ASB_CUDA(cudaMalloc(&table, (size_t)Ns * Ns * sizeof(double)));
        if (backend == OP_FFT) {
            // Love table on the device (boussinesq_kernel.cpp:97-106) at the
            // caller's cell size L / Nl (embedded: offsets up to the compute
            // grid, of which the padded convolution of the block reads |d| < Nl)
            const double h = L / Nl;
            love_table_kernel<<<592, 256>>>(table, Ns, h, 1.0 / (M_PI * E_star));
            ASB_CUDA(cudaGetLastError());
        } else {
            periodic_kernel_table(Nl, Ns, scale, table);
        }
        ASB_SIZE_SWITCH(Ns, KhBuild<NS>::run(*this));
        const size_t nt = (size_t)(Ns + 16) * (Ns + 1);  // widest tiling
        if (supports(true)) {  // no FP64 copy where FP64 applies do not exist
            ASB_CUDA(cudaMalloc(&kh_d, nt * sizeof(double)));
            ASB_CUDA(cudaMemset(kh_d, 0, nt * sizeof(double)));
        }
        ASB_CUDA(cudaMalloc(&kh_f, nt * sizeof(float)));
        ASB_CUDA(cudaMemset(kh_f, 0, nt * sizeof(float)));
    } else {
        const size_t nt = (size_t)(Ns / 2 + 16) * (Ns / 2 + 1);  // widest tiling
        if (supports(true)) ASB_CUDA(cudaMalloc(&psym_d, nt * sizeof(double)));
        ASB_CUDA(cudaMalloc(&psym_f, nt * sizeof(float)));
    }
    for (int dbl = 0; dbl < 2; ++dbl) {
        int rv = 0, cv = 0;
        tuned_variants(kind, dbl, Ns, rv, cv);
        ct[dbl] = 0;  // force the first tiling
        set_variants(dbl != 0, rv, cv);
    }
    ASB_CUDA(cudaDeviceSynchronize());
}

Operator::~Operator() {
    std::lock_guard<std::recursive_mutex> setup(setup_mutex());
    ctx_f.reset();
    ctx_d.reset();
    cudaFree(emb_x);
    cudaFree(emb_y);
    cudaFree(khp_canon);
    cudaFree(khp_d);
    cudaFree(khp_f);
    cudaFree(kh_d);
    cudaFree(kh_f);
    cudaFree(kh_canon);
    cudaFree(psym_d);
    cudaFree(psym_f);
    cudaFree(spec_d);
    cudaFree(spec_f);
    cudaFree(table);
}

int Operator::col_tile(bool dbl, int cv) const {
    int c = 1;
    if (kind == OP_FFT) {
        if (dbl) { ASB_SIZE_SWITCH(Ns, c = FreeImpl<double, NS>::ct(cv, FreeImpl<double, NS>::split(*this))); }
        else { ASB_SIZE_SWITCH(Ns, c = FreeImpl<float, NS>::ct(cv, FreeImpl<float, NS>::split(*this))); }
    } else {
        if (dbl) { ASB_SIZE_SWITCH(Ns, c = PeriodicImpl<double, NS>::ct(cv)); }
        else { ASB_SIZE_SWITCH(Ns, c = PeriodicImpl<float, NS>::ct(cv)); }
    }
    return c;
}

void Operator::set_variants(bool dbl, int rv, int cv) {
    if (rv < 0 || rv >= kVariants || cv < 0 || cv >= kVariants)
        throw Error(-1, "launch variant out of range");
    std::lock_guard<std::recursive_mutex> setup(setup_mutex());
    const int c = col_tile(dbl, cv);
    if (kind == OP_FFT && c != ct[dbl]) {
        // re-tile Kh of this precision for the new column tile width (and
        // the preconditioner's spectrum of an embedded grid)
        k_retile_kh<<<1184, 256>>>(Ns, kh_canon, c, dbl ? kh_d : nullptr, c,
                                   dbl ? nullptr : kh_f);
        if (khp_canon)
            k_retile_kh<<<1184, 256>>>(Ns, khp_canon, c, dbl ? khp_d : nullptr, c,
                                       dbl ? nullptr : khp_f);
        ASB_CUDA(cudaGetLastError());
        ASB_CUDA(cudaDeviceSynchronize());
    }
    if (kind == OP_PERIODIC && c != ct[dbl] && (dbl ? psym_d != nullptr : true)) {
        // the multiplier table of this precision for the new tile width
        const int ncols = (Ns / 2 / c + 1) * c;
        k_periodic_symbol<<<1184, 256>>>(Ns, scale, ncols, c, dbl ? psym_d : nullptr,
                                         dbl ? nullptr : psym_f);
        ASB_CUDA(cudaGetLastError());
        ASB_CUDA(cudaDeviceSynchronize());
    }
    rowv[dbl] = rv;
    colv[dbl] = cv;
    ct[dbl] = c;
    if (ctx_f) ctx_f->invalidate();
    if (ctx_d) ctx_d->invalidate();
}

double Operator::autotune(bool dbl, int reps, int& best_rv, int& best_cv) {
    std::lock_guard<std::recursive_mutex> setup(setup_mutex());
    const long N = (long)Ns * Ns;
    const size_t eb = dbl ? 8 : 4;
    void *x = nullptr, *y = nullptr, *flush = nullptr;
    const size_t fb = 256u << 20;  // > 126 MB L2
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    ASB_CUDA(cudaMalloc(&x, N * eb));
    ASB_CUDA(cudaMalloc(&y, N * eb));
    ASB_CUDA(cudaMalloc(&flush, fb));
    ASB_CUDA(cudaMemset(x, 0, N * eb));
    ASB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    ASB_CUDA(cudaEventCreate(&e0));
    ASB_CUDA(cudaEventCreate(&e1));
    double best = 1e300;
    best_rv = rowv[dbl];
    best_cv = colv[dbl];
    try {
        for (int cv = 0; cv < kVariants; ++cv) {
            for (int rv = 0; rv < kVariants; ++rv) {
                set_variants(dbl, rv, cv);
                matvec(dbl, x, y, s, nullptr);
                matvec(dbl, x, y, s, nullptr);
                double tot = 0.0;
                for (int r = 0; r < reps; ++r) {
                    ASB_CUDA(cudaMemsetAsync(flush, r & 0xff, fb, s));
                    ASB_CUDA(cudaEventRecord(e0, s));
                    matvec(dbl, x, y, s, nullptr);
                    ASB_CUDA(cudaEventRecord(e1, s));
                    ASB_CUDA(cudaEventSynchronize(e1));
                    float ms = 0.f;
                    ASB_CUDA(cudaEventElapsedTime(&ms, e0, e1));
                    tot += ms;
                }
                const double mean = tot / reps;
                if (mean < best) {
                    best = mean;
                    best_rv = rv;
                    best_cv = cv;
                }
            }
        }
    } catch (...) {
        cudaFree(x); cudaFree(y); cudaFree(flush);
        cudaStreamDestroy(s); cudaEventDestroy(e0); cudaEventDestroy(e1);
        throw;
    }
    cudaFree(x);
    cudaFree(y);
    cudaFree(flush);
    cudaStreamDestroy(s);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    set_variants(dbl, best_rv, best_cv);
    record_tuned(kind, dbl, Ns, best_rv, best_cv);
    return best;
}

size_t Operator::spectrum_bytes(bool dbl) const {
    size_t n = 0;
    if (kind == OP_FFT) {
        if (dbl) { ASB_SIZE_SWITCH(Ns, n = FreeImpl<double, NS>::spec_elems(FreeImpl<double, NS>::split(*this)) * sizeof(double2)); }
        else { ASB_SIZE_SWITCH(Ns, n = FreeImpl<float, NS>::spec_elems(FreeImpl<float, NS>::split(*this)) * sizeof(float2)); }
    } else {
        if (dbl) { ASB_SIZE_SWITCH(Ns, n = PeriodicImpl<double, NS>::spec_elems() * sizeof(double2)); }
        else { ASB_SIZE_SWITCH(Ns, n = PeriodicImpl<float, NS>::spec_elems() * sizeof(float2)); }
    }
    return n;
}

void* Operator::spectrum(bool dbl, cudaStream_t) {
    void*& p = dbl ? spec_d : spec_f;
    size_t& nb = dbl ? spec_d_bytes : spec_f_bytes;
    if (!p) {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        nb = spectrum_bytes(dbl);
        ASB_CUDA(cudaMalloc(&p, nb));
        ASB_CUDA(cudaMemset(p, 0, nb));
        ASB_CUDA(cudaDeviceSynchronize());
    }
    return p;
}

size_t Operator::resident_bytes() const {
    size_t n = spec_d_bytes + spec_f_bytes;
    if (kind == OP_FFT) {
        const size_t nt = (size_t)(Ns + 16) * (Ns + 1);
        n += nt * (sizeof(double) + sizeof(float));
        n += (size_t)(Ns + 1) * (Ns + 1) * sizeof(double);  // canonical Kh
        n += (size_t)Ns * Ns * sizeof(double);              // Love table
    } else {
        const size_t nt = (size_t)(Ns / 2 + 16) * (Ns / 2 + 1);  // multiplier tables
        n += nt * ((psym_d ? sizeof(double) : 0) + sizeof(float));
    }
    return n;
}

bool Operator::supports(bool dbl) const {
    bool ok = true;
    if (kind == OP_FFT) {
        if (dbl) { ASB_SIZE_SWITCH(Ns, ok = FreeImpl<double, NS>::kSupported); }
        else { ASB_SIZE_SWITCH(Ns, ok = FreeImpl<float, NS>::kSupported); }
    } else {
        if (dbl) { ASB_SIZE_SWITCH(Ns, ok = PeriodicImpl<double, NS>::kSupported); }
        else { ASB_SIZE_SWITCH(Ns, ok = PeriodicImpl<float, NS>::kSupported); }
    }
    return ok;
}

void Operator::matvec(bool dbl, const void* x, void* y, cudaStream_t s, const int* gate, int B,
                      void* spec_b, const PkState* sc) {
    if (!supports(dbl))
        throw Error(-1, "FP64 applies are not supported above grid_size 8192 (an FP64 row or "
                        "column of 16384 points does not fit one CTA's shared memory); use FP32");
    void* spec = spec_b ? spec_b : spectrum(dbl, s);
    if (kind == OP_FFT) {
        if (dbl) {
            ASB_SIZE_SWITCH(Ns, FreeImpl<double, NS>::matvec(*this, (const double*)x, (double*)y,
                                                             (double2*)spec, s, gate, B, sc));
        } else {
            ASB_SIZE_SWITCH(Ns, FreeImpl<float, NS>::matvec(*this, (const float*)x, (float*)y,
                                                            (float2*)spec, s, gate, B, sc));
        }
    } else {
        if (dbl) {
            ASB_SIZE_SWITCH(Ns, PeriodicImpl<double, NS>::matvec(*this, (const double*)x,
                                                                 (double*)y, (double2*)spec, s,
                                                                 gate, B, sc));
        } else {
            ASB_SIZE_SWITCH(Ns, PeriodicImpl<float, NS>::matvec(*this, (const float*)x,
                                                                (float*)y, (float2*)spec, s,
                                                                gate, B, sc));
        }
    }
}

void Operator::matvec_defect(const double* x, const double* x0, double* y, const double* y0,
                             cudaStream_t s, const int* gate, int B, void* spec_b,
                             const PkState* sc) {
    void* spec = spec_b ? spec_b : spectrum(false, s);
    const long bx = (long)Ns * Ns;
    if (kind == OP_FFT) {
        ASB_SIZE_SWITCH(Ns, FreeImpl<float, NS>::apply(*this, LoadDiffRows{x, x0, NS, bx, sc},
                                                       StoreAddRows{y, y0, NS, bx},
                                                       (float2*)spec, s, gate, B));
    } else {
        ASB_SIZE_SWITCH(Ns, PeriodicImpl<float, NS>::apply(
                                rowv[0], colv[0], LoadDiffRows{x, x0, NS, bx, sc},
                                PeriodicImpl<float, NS>::mult(*this), StoreAddRows{y, y0, NS, bx},
                                (float2*)spec, s, gate, B));
    }
}

void Operator::apply_caller(bool dbl, const void* x, void* y, cudaStream_t s) {
    if (!embedded()) {
        matvec(dbl, x, y, s);
        return;
    }
    const long n = (long)Ns * Ns, nl = (long)Nl * Nl;
    if (!emb_x) {
        std::lock_guard<std::recursive_mutex> setup(setup_mutex());
        ASB_CUDA(cudaMalloc(&emb_x, n * sizeof(double)));
        ASB_CUDA(cudaMalloc(&emb_y, n * sizeof(double)));
    }
    if (dbl) {
        k_embed<double, double><<<embed_grid(n), 256, 0, s>>>(Nl, Ns, 1, (const double*)x,
                                                              (double*)emb_x, 0.0);
        matvec(true, emb_x, emb_y, s);
        k_extract<double, double><<<embed_grid(nl), 256, 0, s>>>(Nl, Ns, 1,
                                                                 (const double*)emb_y, (double*)y);
    } else {
        k_embed<float, float><<<embed_grid(n), 256, 0, s>>>(Nl, Ns, 1, (const float*)x,
                                                            (float*)emb_x, 0.0f);
        matvec(false, emb_x, emb_y, s);
        k_extract<float, float><<<embed_grid(nl), 256, 0, s>>>(Nl, Ns, 1, (const float*)emb_y,
                                                               (float*)y);
    }
    count_launches(2);
    ASB_CUDA(cudaGetLastError());
}

void Operator::ensure_precond_spectrum() {
    if (khp_canon) return;
    if (!embedded() || kind != OP_FFT)
        throw Error(-1, "ensure_precond_spectrum: embedded grids only");
    if (Nl % 2)
        throw Error(-1, "precond 'fourier-fft' on a grid that is not a power of two needs an "
                        "even grid_size (its |k| symbol is not even on an odd torus)");
    std::lock_guard<std::recursive_mutex> setup(setup_mutex());
    double* tab = nullptr;
    const size_t nk = (size_t)(Ns + 1) * (Ns + 1), nt = (size_t)(Ns + 16) * (Ns + 1);
    try {
        ASB_CUDA(cudaMalloc(&tab, (size_t)Ns * Ns * sizeof(double)));
        periodic_kernel_table(Nl, Ns, 0.0, tab, 1);
        ASB_CUDA(cudaMalloc(&khp_canon, nk * sizeof(double)));
        ASB_SIZE_SWITCH(Ns, (void)KhBuild<NS>::build(*this, tab, khp_canon));
        if (supports(true)) {
            ASB_CUDA(cudaMalloc(&khp_d, nt * sizeof(double)));
            ASB_CUDA(cudaMemset(khp_d, 0, nt * sizeof(double)));
            k_retile_kh<<<1184, 256>>>(Ns, khp_canon, ct[1], khp_d, ct[1], nullptr);
        }
        ASB_CUDA(cudaMalloc(&khp_f, nt * sizeof(float)));
        ASB_CUDA(cudaMemset(khp_f, 0, nt * sizeof(float)));
        k_retile_kh<<<1184, 256>>>(Ns, khp_canon, ct[0], nullptr, ct[0], khp_f);
        ASB_CUDA(cudaGetLastError());
        ASB_CUDA(cudaDeviceSynchronize());
    } catch (...) {
        cudaFree(tab);
        cudaFree(khp_canon);
        cudaFree(khp_d);
        cudaFree(khp_f);
        khp_canon = nullptr;
        khp_d = nullptr;
        khp_f = nullptr;
        throw;
    }
    cudaFree(tab);
}

// the full-grid |k| preconditioner of an embedded grid: the masked centred
// residual convolved with the symbol's real-space kernel on the Nl torus by
// the compute grid's padded pipeline, gathered on contact with its contact
// sum (the same load and store as the periodic form)
template <typename T, int NS>
struct EmbeddedFourierImpl {
    static void run(Operator& op, const T* g, const uint8_t* mask, PkState* st, T* z,
                    double* part, cudaStream_t s, const int* gate, int B, void* spec_b) {
        if (!op.khp_canon)
            throw Error(-1, "fourier-fft preconditioner spectrum not built (set-up order)");
        cplx<T>* spec = static_cast<cplx<T>*>(spec_b ? spec_b : op.spectrum(sizeof(T) == 8, s));
        const long bx = (long)NS * NS;
        const T* kh = sizeof(T) == 8 ? (const T*)op.khp_d : (const T*)op.khp_f;
        FreeImpl<T, NS>::apply(op, LoadMaskCentered<T>{g, mask, st, NS, bx},
                               StoreGather<T>{z, mask, NS, st, part, bx, 0.0}, spec, s, gate, B,
                               kh);
    }
};

template <typename T>
void fourier_precond_pk(Operator& op, const T* g, const uint8_t* mask, PkState* st, T* z,
                        double* part, cudaStream_t s, const int* gate, int B, void* spec) {
    if (op.embedded()) {
        ASB_SIZE_SWITCH(op.Ns, EmbeddedFourierImpl<T, NS>::run(op, g, mask, st, z, part, s, gate,
                                                               B, spec));
        return;
    }
    ASB_SIZE_SWITCH(op.Ns, FourierImpl<T, NS>::run(op, g, mask, st, z, part, s, gate, B, spec));
}
template void fourier_precond_pk<float>(Operator&, const float*, const uint8_t*, PkState*, float*,
                                        double*, cudaStream_t, const int*, int, void*);
template void fourier_precond_pk<double>(Operator&, const double*, const uint8_t*, PkState*,
                                         double*, double*, cudaStream_t, const int*, int, void*);

}  // namespace asb
