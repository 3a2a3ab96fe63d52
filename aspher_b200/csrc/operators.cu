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
#include "ops.hpp"
#include "pcg.hpp"
#include "reduce.cuh"

#include <atomic>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

namespace asb {

// ----------------------------------------------------------------------------
// twiddle tables
// ----------------------------------------------------------------------------
namespace {
std::mutex g_tw_mu;
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
        std::lock_guard<std::mutex> lk(g_tw_mu);
        if (!g_tw[dev][0]) build_tw(dev);
    }
    if (L < 1 || L > kMaxTw) throw Error(-1, "twiddle length out of range");
    if (dbl) return static_cast<const double2*>(g_tw[dev][1]) + L;
    return static_cast<const float2*>(g_tw[dev][0]) + L;
}

bool is_pow2(long v) { return v > 0 && (v & (v - 1)) == 0; }

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
__device__ double asinh_diff_dev(double u, double v, double du) {
    if (fabs(u) > 1e150 || fabs(v) > 1e150) return asinh(u) - asinh(v);
    const double su = sqrt(1.0 + u * u), sv = sqrt(1.0 + v * v);
    const double den = u * sv + v * su;
    const double w = (u * v > 0.0 && den != 0.0) ? du * (u + v) / den : u * sv - v * su;
    return asinh(w);
}

__device__ __forceinline__ double love_term(double t, double s1, double s2, double ds) {
    if (t == 0.0) return 0.0;
    const double c = fabs(t);
    return t * asinh_diff_dev(s1 / c, s2 / c, ds / c);
}

__device__ double love_uz_dev(double x, double y, double a, double b) {
    x = fabs(x);
    y = fabs(y);
    const double m = a > b ? a : b;
    const double r2 = x * x + y * y;
    const double sw = 1500.0 * m;
    if (r2 > sw * sw) {
        const double r = sqrt(r2);
        const double A = 4.0 * a * b;
        const double quad = (a * a * (3.0 * x * x - r2) + b * b * (3.0 * y * y - r2)) /
                            (6.0 * r2 * r2);
        return A * (1.0 + quad) / r;
    }
    const double xp = x + a, xm = x - a, yp = y + b, ym = y - b;
    const double da = 2.0 * a, db = 2.0 * b;
    return love_term(xp, yp, ym, db) + love_term(yp, xp, xm, da) +
           love_term(xm, ym, yp, -db) + love_term(ym, xm, xp, -da);
}

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
template <typename T>
struct LoadRealRows {  // z[n] = (x[row*pitch + 2n], x[row*pitch + 2n + 1])
    const T* x;
    int pitch;
    __device__ __forceinline__ cplx<T> operator()(int row, int n) const {
        return *reinterpret_cast<const cplx<T>*>(x + (size_t)row * pitch + 2 * n);
    }
};

template <typename T>
struct StoreRealRows {
    T* y;
    int pitch;
    static constexpr bool kFinish = false;
    __device__ __forceinline__ void operator()(int row, int n, cplx<T> z) const {
        *reinterpret_cast<cplx<T>*>(y + (size_t)row * pitch + 2 * n) = z;
    }
    __device__ void finish(double*) const {}
};

template <typename T>
struct StoreTiled {
    cplx<T>* base;
    int nrows, ct;
    static constexpr bool kFinish = false;
    __device__ __forceinline__ void operator()(int row, int k, cplx<T> X) const {
        base[(size_t)(k / ct) * nrows * ct + (size_t)row * ct + (k % ct)] = X;
    }
    __device__ void finish(double*) const {}
};

template <typename T>
struct LoadTiled {
    const cplx<T>* base;
    int nrows, ct;
    __device__ __forceinline__ cplx<T> operator()(int row, int k) const {
        return base[(size_t)(k / ct) * nrows * ct + (size_t)row * ct + (k % ct)];
    }
};

// Free-space multiplier: real Kh, even-folded in ky, tiled like the spectrum
// with ct columns per tile and Ns+1 rows.
template <typename T>
struct KhMult {
    const T* kh;
    int nk;  // Ns + 1 rows
    int M;   // padded length 2 Ns
    int ct;
    __device__ __forceinline__ cplx<T> operator()(cplx<T> X, int kx, int ky) const {
        const int kf = ky <= (M >> 1) ? ky : M - ky;
        const T w = __ldg(&kh[(size_t)(kx / ct) * nk * ct + (size_t)kf * ct + (kx % ct)]);
        return cscale(X, w);
    }
};

// Periodic multiplier: scale / |m| in FP64, cast to T (periodic_fft_operator.cpp:34-47).
template <typename T>
struct PeriodicMult {
    double scale;
    int Ns;
    __device__ __forceinline__ cplx<T> operator()(cplx<T> X, int kx, int ky) const {
        const int my = ky < (Ns + 1) / 2 ? ky : ky - Ns;
        const double m2 = (double)kx * kx + (double)my * my;
        const T w = m2 > 0.0 ? (T)(scale / sqrt(m2)) : T(0);
        return cscale(X, w);
    }
};

// ---- Kh build functors (FP64) -------------------------------------------------
// Embedded table K(iy, ix) = T(|d(iy)|, |d(ix)|), d(i) = i (i < Ns) or i - M,
// with row/column Ns zero (fft_operator.cpp:31-44), generated on the fly.
struct LoadEmbedded {
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
// Pass B: Kh[(row/ct)][k][row%ct] = Re X / M^2 in FP64 and FP32 copies.
struct StoreRealTracked {
    double* out_t;  // pass A: transposed real, (Ns+1) x M
    int M;
    double* kh_d;   // pass B
    float* kh_f;
    int nk, ct_d, ct_f;
    double norm;
    unsigned long long* maxbits;  // [0] = max|Im|, [1] = max|Re| (as bit patterns)
    static constexpr bool kFinish = true;
    mutable double mi, mr;
    __device__ __forceinline__ void operator()(int row, int k, double2 X) const {
        if (out_t) {
            out_t[(size_t)k * M + row] = X.x;
        } else {
            const double v = X.x * norm;
            kh_d[(size_t)(row / ct_d) * nk * ct_d + (size_t)k * ct_d + (row % ct_d)] = v;
            kh_f[(size_t)(row / ct_f) * nk * ct_f + (size_t)k * ct_f + (row % ct_f)] = (float)v;
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

// ----------------------------------------------------------------------------
// per-size implementation
// ----------------------------------------------------------------------------
template <typename T, int NS>
struct FreeImpl {
    static constexpr int LR = NS, LC = 2 * NS;
    static constexpr int CT = col_ct<T>(LC, LR);
    static constexpr int NT = LR / CT + 1;  // tiles over Ns+1 columns

    static size_t spec_elems() { return (size_t)NT * NS * CT; }

    static void matvec(const Operator& op, const T* x, T* y, cplx<T>* spec, cudaStream_t s,
                       const int* gate) {
        if constexpr (col_smem<T>(LC, CT) > 227 * 1024) {
            throw Error(-1, "free-space FP64 apply at grid_size 8192 is not supported (the "
                            "16384-point FP64 column does not fit one CTA's shared memory); "
                            "use FP32 or grid_size <= 4096");
        } else {
        constexpr int rb = row_rb<T>(LR);
        constexpr int rthreads = rb * (LR / rpt_for(LR));
        constexpr int rsm = row_smem<T>(LR);
        const int rgrid = (NS + rb - 1) / rb;
        auto kf = row_fwd_kernel<T, LR, true, LoadRealRows<T>, StoreTiled<T>>;
        smem_optin((const void*)kf, rsm);
        kf<<<rgrid, rthreads, rsm, s>>>(LoadRealRows<T>{x, NS}, StoreTiled<T>{spec, NS, CT}, NS,
                                        tw<T>(LR), tw<T>(2 * LR), gate);
        constexpr int cthreads = CT * (LC / rpt_for(LC));
        constexpr int csm = col_smem<T>(LC, CT);
        auto kc = col_kernel<T, LC, CT, true, KhMult<T>>;
        smem_optin((const void*)kc, csm);
        const T* kh = sizeof(T) == 8 ? (const T*)op.kh_d : (const T*)op.kh_f;
        kc<<<NT, cthreads, csm, s>>>(spec, NS, KhMult<T>{kh, NS + 1, LC, CT}, tw<T>(LC), gate);
        auto ki = row_inv_kernel<T, LR, true, LoadTiled<T>, StoreRealRows<T>>;
        smem_optin((const void*)ki, rsm);
        ki<<<rgrid, rthreads, rsm, s>>>(LoadTiled<T>{spec, NS, CT}, StoreRealRows<T>{y, NS}, NS,
                                        tw<T>(LR), tw<T>(2 * LR), gate);
        count_launches(3);
        ASB_CUDA(cudaGetLastError());
        }
    }
};

template <typename T, int NS>
struct PeriodicImpl {
    static constexpr int LR = NS / 2, LC = NS;
    static constexpr int CT = col_ct<T>(LC, LR);
    static constexpr int NT = LR / CT + 1;

    static size_t spec_elems() { return (size_t)NT * NS * CT; }

    template <class Mult>
    static void apply_mult(const T* x, T* y, cplx<T>* spec, Mult mult, cudaStream_t s,
                           const int* gate) {
        constexpr int rb = row_rb<T>(LR);
        constexpr int rthreads = rb * (LR / rpt_for(LR));
        constexpr int rsm = row_smem<T>(LR);
        const int rgrid = (NS + rb - 1) / rb;
        auto kf = row_fwd_kernel<T, LR, false, LoadRealRows<T>, StoreTiled<T>>;
        smem_optin((const void*)kf, rsm);
        kf<<<rgrid, rthreads, rsm, s>>>(LoadRealRows<T>{x, NS}, StoreTiled<T>{spec, NS, CT}, NS,
                                        tw<T>(LR), tw<T>(2 * LR), gate);
        constexpr int cthreads = CT * (LC / rpt_for(LC));
        constexpr int csm = col_smem<T>(LC, CT);
        auto kc = col_kernel<T, LC, CT, false, Mult>;
        smem_optin((const void*)kc, csm);
        kc<<<NT, cthreads, csm, s>>>(spec, NS, mult, tw<T>(LC), gate);
        auto ki = row_inv_kernel<T, LR, false, LoadTiled<T>, StoreRealRows<T>>;
        smem_optin((const void*)ki, rsm);
        ki<<<rgrid, rthreads, rsm, s>>>(LoadTiled<T>{spec, NS, CT}, StoreRealRows<T>{y, NS}, NS,
                                        tw<T>(LR), tw<T>(2 * LR), gate);
        count_launches(3);
        ASB_CUDA(cudaGetLastError());
    }

    static void matvec(const Operator& op, const T* x, T* y, cplx<T>* spec, cudaStream_t s,
                       const int* gate) {
        apply_mult(x, y, spec, PeriodicMult<T>{op.scale, NS}, s, gate);
    }
};


// ----------------------------------------------------------------------------
// full-grid |k| preconditioner (reference: src/fourier_precond.cpp:12-116)
// ----------------------------------------------------------------------------
template <typename T>
struct LoadMaskCentered {  // contact ? g - T(gsum/ng) : 0, pairwise
    const T* g;
    const uint8_t* mask;
    const PkState* st;
    int pitch;
    __device__ __forceinline__ cplx<T> operator()(int row, int n) const {
        const int nc = st->nc;
        const T gm = nc ? (T)(st->gcs / nc) : T(0);
        const size_t i = (size_t)row * pitch + 2 * n;
        const cplx<T> v = *reinterpret_cast<const cplx<T>*>(g + i);
        const uchar2 m = *reinterpret_cast<const uchar2*>(mask + i);
        return mk<T>(m.x ? (T)(v.x - gm) : T(0), m.y ? (T)(v.y - gm) : T(0));
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
    T* z;
    const uint8_t* mask;
    int pitch;
    PkState* st;
    double* part;
    static constexpr bool kFinish = true;
    double zs;
    __device__ __forceinline__ void operator()(int row, int n, cplx<T> v) {
        const size_t i = (size_t)row * pitch + 2 * n;
        const uchar2 m = *reinterpret_cast<const uchar2*>(mask + i);
        *reinterpret_cast<cplx<T>*>(z + i) = mk<T>(m.x ? v.x : T(0), m.y ? v.y : T(0));
        if (m.x) zs += (double)v.x;
        if (m.y) zs += (double)v.y;
    }
    __device__ void finish(double*) {
        double a[1] = {zs};
        const int kinds[1] = {0};
        if (grid_reduce_last<1>(a, kinds, part, &st->counter[11]) && threadIdx.x == 0) {
            const int nc = st->nc;
            st->zmean = nc ? (double)(T)(a[0] / nc) : 0.0;
            st->pc++;
        }
    }
};

template <typename T, int NS>
struct FourierImpl {
    using PI = PeriodicImpl<T, NS>;
    static void run(Operator& op, const T* g, const uint8_t* mask, PkState* st, T* z,
                    double* part, cudaStream_t s, const int* gate) {
        constexpr int LR = PI::LR, LC = PI::LC, CT = PI::CT, NT = PI::NT;
        cplx<T>* spec = static_cast<cplx<T>*>(op.spectrum(sizeof(T) == 8, s));
        constexpr int rb = row_rb<T>(LR);
        constexpr int rthreads = rb * (LR / rpt_for(LR));
        constexpr int rsm = row_smem<T>(LR);
        const int rgrid = (NS + rb - 1) / rb;
        auto kf = row_fwd_kernel<T, LR, false, LoadMaskCentered<T>, StoreTiled<T>>;
        smem_optin((const void*)kf, rsm);
        kf<<<rgrid, rthreads, rsm, s>>>(LoadMaskCentered<T>{g, mask, st, NS},
                                        StoreTiled<T>{spec, NS, CT}, NS, tw<T>(LR),
                                        tw<T>(2 * LR), gate);
        constexpr int cthreads = CT * (LC / rpt_for(LC));
        constexpr int csm = col_smem<T>(LC, CT);
        auto kc = col_kernel<T, LC, CT, false, FourierMult<T>>;
        smem_optin((const void*)kc, csm);
        const float norm = 1.0f / ((float)NS * (float)NS);
        kc<<<NT, cthreads, csm, s>>>(spec, NS, FourierMult<T>{NS, norm}, tw<T>(LC), gate);
        auto ki = row_inv_kernel<T, LR, false, LoadTiled<T>, StoreGather<T>>;
        smem_optin((const void*)ki, rsm);
        ki<<<rgrid, rthreads, rsm, s>>>(LoadTiled<T>{spec, NS, CT},
                                        StoreGather<T>{z, mask, NS, st, part, 0.0}, NS, tw<T>(LR),
                                        tw<T>(2 * LR), gate);
        count_launches(3);
        ASB_CUDA(cudaGetLastError());
    }
};

// Kh build for the free-space operator of size NS (FP64).
template <int NS>
struct KhBuild {
    static void run(Operator& op) {
        constexpr int LR = NS, M = 2 * NS;
        constexpr int CTD = FreeImpl<double, NS>::CT, CTF = FreeImpl<float, NS>::CT;
        op.ct_d = CTD;
        op.ct_f = CTF;
        const size_t nkd = (size_t)(NS / CTD + 1) * (NS + 1) * CTD;
        const size_t nkf = (size_t)(NS / CTF + 1) * (NS + 1) * CTF;
        ASB_CUDA(cudaMalloc(&op.kh_d, nkd * sizeof(double)));
        ASB_CUDA(cudaMalloc(&op.kh_f, nkf * sizeof(float)));
        ASB_CUDA(cudaMemset(op.kh_d, 0, nkd * sizeof(double)));
        ASB_CUDA(cudaMemset(op.kh_f, 0, nkf * sizeof(float)));
        double* yt = nullptr;
        unsigned long long* mx = nullptr;
        ASB_CUDA(cudaMalloc(&yt, (size_t)(NS + 1) * M * sizeof(double)));
        ASB_CUDA(cudaMalloc(&mx, 4 * sizeof(unsigned long long)));
        ASB_CUDA(cudaMemset(mx, 0, 4 * sizeof(unsigned long long)));
        constexpr int rb = row_rb<double>(LR);
        constexpr int rthreads = rb * (LR / rpt_for(LR));
        constexpr int rsm = row_smem<double>(LR);
        auto k = row_fwd_kernel<double, LR, false, LoadEmbedded, StoreRealTracked>;
        smem_optin((const void*)k, rsm);
        // pass A over the M rows of the embedded table
        StoreRealTracked sa{yt, M, nullptr, nullptr, 0, 0, 0, 0.0, mx, 0.0, 0.0};
        k<<<(M + rb - 1) / rb, rthreads, rsm>>>(LoadEmbedded{op.table, NS, M}, sa, M,
                                                tw<double>(LR), tw<double>(2 * LR), nullptr);
        ASB_CUDA(cudaGetLastError());
        // pass B over the Ns+1 rows of the transposed buffer (each M long)
        auto k2 = row_fwd_kernel<double, LR, false, LoadRealRows<double>, StoreRealTracked>;
        smem_optin((const void*)k2, rsm);
        StoreRealTracked sb{nullptr, M, op.kh_d, op.kh_f, NS + 1, CTD, CTF,
                            1.0 / ((double)M * (double)M), mx + 2, 0.0, 0.0};
        k2<<<(NS + 1 + rb - 1) / rb, rthreads, rsm>>>(LoadRealRows<double>{yt, M}, sb, NS + 1,
                                                      tw<double>(LR), tw<double>(2 * LR),
                                                      nullptr);
        ASB_CUDA(cudaGetLastError());
        unsigned long long h[4];
        ASB_CUDA(cudaMemcpy(h, mx, sizeof(h), cudaMemcpyDeviceToHost));
        ASB_CUDA(cudaFree(yt));
        ASB_CUDA(cudaFree(mx));
        double v[4];
        for (int i = 0; i < 4; ++i) std::memcpy(&v[i], &h[i], sizeof(double));
        const double ra = v[1] > 0 ? v[0] / v[1] : 0.0;
        const double rbt = v[3] > 0 ? v[2] / v[3] : 0.0;
        op.max_im_ratio = ra > rbt ? ra : rbt;
        // fft_operator.cpp:57-60: the embedding is even, so the spectrum is real
        if (v[0] > 1e-10 * v[1] || v[2] > 1e-10 * v[3])
            throw Error(-3, "FFTOperator: kernel spectrum has a non-negligible imaginary "
                            "part; wrap-around embedding is broken");
    }
};

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
        default: throw Error(-1, "grid_size must be a power of two in [16, 8192]"); \
    }

Operator::Operator(int kind_, int Ns_, double L_, double E_)
    : kind(kind_), Ns(Ns_), L(L_), E_star(E_) {
    if (kind != OP_FFT && kind != OP_PERIODIC) throw Error(-1, "unknown operator kind");
    if (!is_pow2(Ns) || Ns < 16 || Ns > 8192)
        throw Error(-1, "grid_size must be a power of two in [16, 8192]");
    if (!(L > 0.0) || !std::isfinite(L)) throw Error(-1, "domain_size must be positive");
    if (!(E_star > 0.0) || !std::isfinite(E_star)) throw Error(-1, "E_star must be positive");
    ASB_CUDA(cudaGetDevice(&device));
    (void)tw_table(false, 2);
    if (kind == OP_PERIODIC) {
        scale = L / (M_PI * E_star * (double)Ns * Ns);
        return;
    }
    // Love table on the device (boussinesq_kernel.cpp:97-106)
    ASB_CUDA(cudaMalloc(&table, (size_t)Ns * Ns * sizeof(double)));
    const double h = L / Ns;
    love_table_kernel<<<592, 256>>>(table, Ns, h, 1.0 / (M_PI * E_star));
    ASB_CUDA(cudaGetLastError());
    ASB_SIZE_SWITCH(Ns, KhBuild<NS>::run(*this));
    ASB_CUDA(cudaDeviceSynchronize());
}

Operator::~Operator() {
    ctx_f.reset();
    ctx_d.reset();
    cudaFree(kh_d);
    cudaFree(kh_f);
    cudaFree(spec_d);
    cudaFree(spec_f);
    cudaFree(table);
}

size_t Operator::spectrum_bytes(bool dbl) const {
    size_t n = 0;
    if (kind == OP_FFT) {
        if (dbl) { ASB_SIZE_SWITCH(Ns, n = FreeImpl<double, NS>::spec_elems() * sizeof(double2)); }
        else { ASB_SIZE_SWITCH(Ns, n = FreeImpl<float, NS>::spec_elems() * sizeof(float2)); }
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
        n += (size_t)(Ns / ct_d + 1) * (Ns + 1) * ct_d * sizeof(double);
        n += (size_t)(Ns / ct_f + 1) * (Ns + 1) * ct_f * sizeof(float);
        n += (size_t)Ns * Ns * sizeof(double);
    }
    return n;
}

void Operator::matvec(bool dbl, const void* x, void* y, cudaStream_t s, const int* gate) {
    void* spec = spectrum(dbl, s);
    if (kind == OP_FFT) {
        if (dbl) {
            ASB_SIZE_SWITCH(Ns, FreeImpl<double, NS>::matvec(*this, (const double*)x, (double*)y,
                                                             (double2*)spec, s, gate));
        } else {
            ASB_SIZE_SWITCH(Ns, FreeImpl<float, NS>::matvec(*this, (const float*)x, (float*)y,
                                                            (float2*)spec, s, gate));
        }
    } else {
        if (dbl) {
            ASB_SIZE_SWITCH(Ns, PeriodicImpl<double, NS>::matvec(*this, (const double*)x,
                                                                 (double*)y, (double2*)spec, s,
                                                                 gate));
        } else {
            ASB_SIZE_SWITCH(Ns, PeriodicImpl<float, NS>::matvec(*this, (const float*)x,
                                                                (float*)y, (float2*)spec, s,
                                                                gate));
        }
    }
}

template <typename T>
void fourier_precond_pk(Operator& op, const T* g, const uint8_t* mask, PkState* st, T* z,
                        double* part, cudaStream_t s, const int* gate) {
    ASB_SIZE_SWITCH(op.Ns, FourierImpl<T, NS>::run(op, g, mask, st, z, part, s, gate));
}
template void fourier_precond_pk<float>(Operator&, const float*, const uint8_t*, PkState*, float*,
                                        double*, cudaStream_t, const int*);
template void fourier_precond_pk<double>(Operator&, const double*, const uint8_t*, PkState*,
                                         double*, double*, cudaStream_t, const int*);

}  // namespace asb
