// Internal (non-ABI) declarations shared by the translation units of
// libaspher_b200.so: the operator objects, the twiddle tables and the error
// plumbing behind aspher_last_error().
#pragma once

#include <cuda_runtime.h>

#include "pk_state.hpp"

#include <cstddef>
#include <cstdint>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>

namespace asb {

// Exceptions never cross the C ABI: every entry point catches and converts.
struct Error : std::runtime_error {
    int code;
    Error(int c, const std::string& m) : std::runtime_error(m), code(c) {}
};

#define ASB_CUDA(call)                                                           \
    do {                                                                         \
        cudaError_t e_ = (call);                                                 \
        if (e_ != cudaSuccess)                                                   \
            throw ::asb::Error(-2, std::string(#call) + ": " + cudaGetErrorString(e_)); \
    } while (0)

void set_last_error(const std::string& m);

// Kernel launches issued by this library (aspher_launch_count()).
void count_launches(long n);
long long launch_count();

// Cached solver state attached to an operator (see pcg.cu).
struct SolverCtxBase {
    virtual ~SolverCtxBase() = default;
    virtual size_t bytes() const = 0;
    // drop captured graphs (they bake in launch variants and layouts)
    virtual void invalidate() = 0;
};

// exp(-2 pi i k / L), k < L, for every power of two L <= kMaxTw, on the
// current device; tw_f(L)/tw_d(L) return the length-L table.
constexpr int kMaxTw = 32768;
const void* tw_table(bool dbl, int L);
template <typename T> inline const typename std::conditional<sizeof(T) == 4, float2, double2>::type*
tw(int L) {
    return static_cast<const typename std::conditional<sizeof(T) == 4, float2, double2>::type*>(
        tw_table(sizeof(T) == 8, L));
}

enum OpKind : int { OP_FFT = 0, OP_PERIODIC = 1 };
// operator creation flags (aspher_op_create_ex): cross-check forms
enum OpFlags : int { OPF_SPLIT_COLUMNS = 1, OPF_SPLIT_KH = 2 };

// smallest grid with the split free-space column pass (two length-Ns halves
// of the length-2Ns column; required for FP64 at Ns = 8192)
constexpr int kSplitMin = 256;
// largest grid; above kMaxVariantNs the pass kernels run launch variant 0
// only, and only FP32 (an FP64 row or half column of 16384 points does not
// fit one CTA's shared memory)
constexpr int kMaxNs = 16384;
constexpr int kMaxVariantNs = 8192;

bool is_pow2(long v);

// launch variants chosen for (kind, precision, Ns): the autotuned entry of
// this process if any, else the built-in default
void tuned_variants(int kind, int dbl, int Ns, int& rv, int& cv);

// Process-wide lock for work that must not overlap a CUDA-graph capture in
// another host thread: graph capture itself and the set-up / tear-down calls
// that synchronise the device (cudaMalloc / cudaMemset / cudaFree /
// cudaDeviceSynchronize / blocking copies).  Recursive: set-up paths nest.
std::recursive_mutex& setup_mutex();

// Opt into >48 KB dynamic shared memory once per kernel per device.
void smem_optin(const void* func, int bytes);

struct Operator {
    // the compute grid: a power of two in [16, 16384] and the pipeline
    // (free-space padded or periodic) that every kernel of this library sees
    int kind = OP_FFT;
    int Ns = 0;
    double L = 1.0, E_star = 1.0;
    // the caller's grid side and backend.  Equal to Ns / kind unless the
    // caller's side is not a power of two in [16, 16384]: the operator then
    // runs EMBEDDED, its Nl x Nl cells the top-left block of an Ns x Ns
    // free-space pipeline (Ns the next power of two, at least 16) whose
    // kernel table holds the caller's operator at every offset |d| < Nl:
    // the Love table at the caller's cell size (backend fft: the padded
    // convolution of the block is the free-space operator of the Nl grid),
    // or the real-space kernel of the periodic symbol on the Nl torus
    // (backend periodic: a circulant on the Nl torus is a linear
    // convolution with that kernel over offsets |d| < Nl)
    int Nl = 0;
    int backend = OP_FFT;
    bool embedded() const { return Nl != Ns || backend != kind; }
    // embedded: Ns*Ns scratch fields of the caller-facing apply (lazy)
    void* emb_x = nullptr;
    void* emb_y = nullptr;
    // caller-facing apply: x, y hold Nl*Nl values (embedded: copied into the
    // compute grid's block and back; otherwise matvec)
    void apply_caller(bool dbl, const void* x, void* y, cudaStream_t s);
    // embedded grids (even Nl) with the full-grid |k| preconditioner: the
    // spectrum of its real-space kernel on the Nl torus, canonical and tiled
    // like Kh; built by ensure_precond_spectrum() (set-up, not under capture)
    double* khp_canon = nullptr;
    double* khp_d = nullptr;
    float* khp_f = nullptr;
    void ensure_precond_spectrum();
    int device = 0;
    // free space: real half spectrum Kh (1/M^2 folded in), rows ky in [0, Ns]
    // only (Kh is even in ky): canonical [ky][kx] FP64, plus FP64 / FP32
    // copies tiled for the active column tile width of each precision
    double* kh_canon = nullptr;
    double* kh_d = nullptr;
    float* kh_f = nullptr;
    // periodic (power-of-two grid): the multiplier scale / |m| over
    // kx in [0, Ns/2] and |m_y| in [0, Ns/2], evaluated in FP64 and rounded
    // to each precision once, tiled like Kh for the active column tile width
    double* psym_d = nullptr;
    float* psym_f = nullptr;
    double max_im_ratio = 0.0;
    // launch variants per precision [F32, F64] and the column tile width
    // (half-spectrum layout) they imply
    int rowv[2] = {0, 0}, colv[2] = {0, 0}, ct[2] = {0, 0};
    // free space: the column pass as two half-length transforms even where
    // the full column fits one CTA (creation flag ASPHER_OPF_SPLIT_COLUMNS,
    // for cross-checks of the form Ns = 8192 FP64 needs)
    bool split_cols = false;
    // free space: the FP64 Kh build from even / odd row samples even where a
    // row fits one CTA (creation flag ASPHER_OPF_SPLIT_KH, for cross-checks)
    bool split_kh = false;
    // periodic: symbol scale L / (pi E* Ns^2)
    double scale = 0.0;
    // scratch half spectra per precision (lazily sized)
    void* spec_d = nullptr;
    void* spec_f = nullptr;
    size_t spec_d_bytes = 0, spec_f_bytes = 0;
    // Love table (free space only), kept for tests/diagnostics
    double* table = nullptr;
    // solver contexts per precision (workspace + loop graph), built lazily
    std::shared_ptr<SolverCtxBase> ctx_f, ctx_d;

    Operator(int kind, int Ns, double L, double E_star, int flags = 0);
    ~Operator();
    Operator(const Operator&) = delete;
    Operator& operator=(const Operator&) = delete;

    // u = S x on `stream`; x, y device arrays of Ns*Ns values of the dtype.
    // gate: optional device int; when nonzero at kernel start, kernels return.
    // Batched (B > 1): x, y hold B fields back to back, spec_b a spectrum
    // scratch of B * spectrum_bytes(dbl), and gate[b * kGateStride] gates
    // instance b.
    // sc (optional): x is a PK loop's pressure with a pending load rescale in
    // sc[b] (PkState::scale / scale_add), applied as x is loaded.
    void matvec(bool dbl, const void* x, void* y, cudaStream_t s, const int* gate = nullptr,
                int B = 1, void* spec_b = nullptr, const PkState* sc = nullptr);
    // Defect-corrected FP64 apply: y = y0 + S_32(x - x0) with x, x0, y, y0
    // FP64 fields (x0, y0 optional) and the transform in FP32.  With
    // y0 = S x0 exact, the result carries the FP32 rounding of S only on the
    // difference x - x0, i.e. FP64-level accuracy while x stays near x0.
    // Batched as matvec (spec_b: B * spectrum_bytes(false) at least).
    void matvec_defect(const double* x, const double* x0, double* y, const double* y0,
                       cudaStream_t s, const int* gate = nullptr, int B = 1,
                       void* spec_b = nullptr, const PkState* sc = nullptr);
    void* spectrum(bool dbl, cudaStream_t s);
    int col_tile(bool dbl, int cv) const;
    void set_variants(bool dbl, int rv, int cv);
    // times every (row, column) variant pair (reps applies each, L2 flushed),
    // keeps and records (process-wide) the fastest; returns its mean ms
    double autotune(bool dbl, int reps, int& best_rv, int& best_cv);
    size_t spectrum_bytes(bool dbl) const;
    // whether applies of this precision exist at this size (false only for
    // FP64 above 8192); checked before any allocation of that precision
    bool supports(bool dbl) const;
    size_t resident_bytes() const;
};

// Full-grid |k| preconditioner (FourierPreconditioner) on the Ns periodic grid.
// g is centred by gmean (device scalar, already in T), masked by contact,
// transformed, multiplied by |k|/Ns^2 and gathered on contact into z.
// The contact sum of z (double) goes to *zsum_out via per-block partials and
// a last-block reduction (deterministic); counter must be zero on entry.
void fourier_precond_apply(Operator& op_shape_src, bool dbl, const void* g,
                           const uint8_t* contact, const double* gmean,
                           void* z, double* zsum_out, double* partials,
                           unsigned* counter, cudaStream_t s, const int* gate);

}  // namespace asb
