// Row and column pass kernels of the 2-D real transforms.
//
// A 2-D r2c/c2r pair over an (nrows x 2*LR) real grid is split as:
//   row_fwd : per row, the real FFT of length 2*LR via a length-LR complex
//             FFT of z[n] = x[2n] + i x[2n+1] and the usual split step,
//             producing the LR+1 half-spectrum columns;
//   col     : per column, forward FFT of length LC, pointwise multiplier,
//             inverse FFT (fused: the spectrum never leaves the CTA);
//   row_inv : per row, the inverse split step and a length-LR complex FFT.
// PAD=true is the zero-padded (Hockney) case of the free-space operator:
// rows hold Ns real values padded to 2*Ns (so half of z is zero and those
// registers are never loaded), and columns hold Ns values padded to LC=2*Ns
// of which only the first Ns outputs are kept.
//
// The half spectrum lives in HBM in a column-tiled layout:
//   elem(row, k) = base[(k / ct) * nrows * ct + row * ct + (k % ct)]
// so a column CTA streams one contiguous tile and a row CTA of RB rows
// touches RB*ct contiguous elements per tile.
//
// Batched solves launch every kernel with gridDim.y = instances; the load /
// store functors offset their pointers by blockIdx.y times a batch stride,
// and instance b's spectrum is the b-th block of gridDim.x column tiles.
//
// Launch shapes are variants (V = 0..kVariants-1) trading registers per
// thread (RPT elements, radix <= RPT), CTA size and CTAs per SM; the
// operator picks one row variant and one column variant per size and
// precision (a default table, or the autotuner in operators.cu).
#pragma once

#include <type_traits>

#include "fft_block.cuh"
#include "pk_state.hpp"

namespace asb {

constexpr int kVariants = 4;
// Batched launches (gridDim.y = instances) read instance b's gate at
// gate[b * kGateStride]: the gates live in consecutive PkState records.
constexpr int kGateStride = (int)(sizeof(PkState) / sizeof(int));
static_assert(sizeof(PkState) % sizeof(int) == 0, "PkState must be a whole number of ints");
constexpr int kSmemPerSM = 227 * 1024;

template <typename T>
struct TiledSpec {
    cplx<T>* base;
    int nrows;
    int ct;
    __device__ __forceinline__ size_t idx(int row, int k) const {
        return (size_t)(k / ct) * nrows * ct + (size_t)row * ct + (k % ct);
    }
};

// ---- variant tables -----------------------------------------------------------------
// Row kernels.  FP32: V0 RPT16/512 thr/1 CTA, V1 RPT16/256/2, V2 RPT8/256/3,
// V3 RPT8/512/2.  FP64: V0 RPT16/512/1, V1 RPT8/256/2, V2 RPT8/256/3,
// V3 RPT8/512/1.
template <typename T>
__host__ __device__ constexpr int row_rpt(int LR, int v) {
    int want = sizeof(T) == 4 ? ((v <= 1) ? 16 : 8) : (v == 0 ? 16 : 8);
    if (want < LR / 1024) want = LR / 1024;  // at most 1024 threads per transform
    return LR < want ? LR : want;
}
template <typename T>
__host__ __device__ constexpr int row_target_threads(int v) {
    return (v == 0 || v == 3) ? 512 : 256;
}
template <typename T>
__host__ __device__ constexpr int row_minb_req(int v) {
    return sizeof(T) == 4 ? (v == 0 ? 1 : (v == 2 ? 3 : 2)) : (v == 1 ? 2 : (v == 2 ? 3 : 1));
}
template <typename T>
__host__ __device__ constexpr int row_rb_v(int LR, int v) {
    const int tt = LR / row_rpt<T>(LR, v);
    int rb = row_target_threads<T>(v) / tt;
    if (rb < 1) rb = 1;
    if (rb > 16) rb = 16;
    const int per_row = sm_len(LR + 1) * (int)sizeof(cplx<T>);
    const int mb = row_minb_req<T>(v);
    while (rb > 1 && rb * per_row * mb > kSmemPerSM) rb >>= 1;
    return rb;
}
template <typename T>
__host__ __device__ constexpr int row_threads(int LR, int v) {
    return row_rb_v<T>(LR, v) * (LR / row_rpt<T>(LR, v));
}
template <typename T>
__host__ __device__ constexpr int row_smem_v(int LR, int v) {
    return row_rb_v<T>(LR, v) * sm_len(LR + 1) * (int)sizeof(cplx<T>);
}
template <typename T>
__host__ __device__ constexpr int row_minb(int LR, int v) {
    int mb = row_minb_req<T>(v);
    while (mb > 1 && mb * row_smem_v<T>(LR, v) > kSmemPerSM) --mb;
    while (mb > 1 && mb * row_threads<T>(LR, v) > 2048) --mb;
    return mb;
}

// Row forward of a zero-padded transform (FP32, variant 1): up to four CTAs
// per SM at 64 registers (1024 / threads of them) instead of two.  Its
// input is half a row and its full groups store with fixed strides, so the
// register budget suffices; measured at Ns=2048 on B200: 24.4 -> 22.3 us.
// The row inverse and the unpadded (staged) forward keep the variant's CTAs
// per SM: both measured slower at four.
template <typename T, int LR, bool PAD, int V>
__host__ __device__ constexpr int row_fwd_minb() {
    int mb = row_minb<T>(LR, V);
    if (PAD && sizeof(T) == 4 && V == 1) {
        int want = 1024 / row_threads<T>(LR, V);
        if (want > 4) want = 4;
        while (want > mb && want * row_smem_v<T>(LR, V) > kSmemPerSM) --want;
        if (want > mb) mb = want;
    }
    return mb;
}

// Column kernel.  FP32: V0 RPT16/<=512 thr/1, V1 RPT16/<=256/2, V2 RPT8/<=512/2,
// V3 RPT8/<=256/3.  FP64: V0 RPT16/<=512/1, V1 RPT8/<=256/2, V2 RPT8/<=512/1,
// V3 RPT8/<=256/3.
template <typename T>
__host__ __device__ constexpr int col_rpt(int LC, int v) {
    int want = sizeof(T) == 4 ? (v <= 1 ? 16 : 8) : (v == 0 ? 16 : 8);
    if (want < LC / 1024) want = LC / 1024;  // at most 1024 threads per transform
    return LC < want ? LC : want;
}
template <typename T>
__host__ __device__ constexpr int col_max_threads(int v) {
    return (v == 0 || v == 2) ? 512 : 256;
}
template <typename T>
__host__ __device__ constexpr int col_minb_req(int v) {
    return sizeof(T) == 4 ? (v == 0 ? 1 : (v == 3 ? 3 : 2)) : (v == 1 ? 2 : (v == 3 ? 3 : 1));
}
template <typename T>
__host__ __device__ constexpr int col_ct_v(int LC, int ncols_minus1, int v) {
    const int tt = LC / col_rpt<T>(LC, v);
    const int mb = col_minb_req<T>(v);
    int ct = 16;
    while (ct > 1 && (ct * tt > col_max_threads<T>(v) ||
                      (ct * sm_len(LC) + ct) * (int)sizeof(cplx<T>) * mb > kSmemPerSM ||
                      ct > ncols_minus1))
        ct >>= 1;
    return ct;
}
template <typename T>
__host__ __device__ constexpr int col_smem(int LC, int ct) {
    return (ct * sm_len(LC) + ct) * (int)sizeof(cplx<T>);
}
template <typename T>
__host__ __device__ constexpr int col_threads(int LC, int ncm1, int v) {
    return col_ct_v<T>(LC, ncm1, v) * (LC / col_rpt<T>(LC, v));
}
template <typename T>
__host__ __device__ constexpr int col_minb(int LC, int ncm1, int v) {
    int mb = col_minb_req<T>(v);
    const int sm = col_smem<T>(LC, col_ct_v<T>(LC, ncm1, v));
    while (mb > 1 && mb * sm > kSmemPerSM) --mb;
    while (mb > 1 && mb * col_threads<T>(LC, ncm1, v) > 2048) --mb;
    return mb;
}
// does a column of length LC fit one CTA at all (variant-independent floor)
template <typename T>
__host__ __device__ constexpr bool col_fits(int LC) {
    return col_smem<T>(LC, 1) <= kSmemPerSM;
}

// ---- software pipeline ----------------------------------------------------------
// When the input of a unit (a row group or a column tile) is a plain
// contiguous block (raw rows, tiled spectrum chunks, a column tile) and a
// staging buffer fits beside the FFT workspace, the pass kernel is
// persistent -- a CTA walks units blockIdx.x, blockIdx.x + gridDim.x, ... --
// and the next unit's input is copied global -> shared with cp.async while
// the current unit is being transformed, so the load latency of one unit hides behind the arithmetic
// of the previous one.  The waits are the hardware's own (cp.async.wait_all):
// no software spin.  Staging is used for the unpadded transforms only: on
// B200 it sped the periodic applies up by 8-16 % (Ns 2048-4096) but slowed
// the zero-padded free-space ones (whose staged inputs are half empty and
// whose larger shared-memory footprint costs resident CTAs).  Unstaged
// kernels process one unit per CTA: the loop would cost registers (the
// 4096-point FP32 column kernel spilled with it).
__host__ __device__ constexpr int align16(int b) { return (b + 15) & ~15; }

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() {
    asm volatile("cp.async.commit_group;\n" ::: "memory");
}
__device__ __forceinline__ void cp_async_wait_all() {
    asm volatile("cp.async.wait_all;\n" ::: "memory");
}
// one complex element global -> shared (8 or 16 bytes)
template <typename T>
__device__ __forceinline__ void cp_async_cplx(cplx<T>* smem, const cplx<T>* gmem) {
    if constexpr (sizeof(cplx<T>) == 16) cp_async16(smem, gmem);
    else cp_async8(smem, gmem);
}

// Row forward: staging of RB raw rows (Ns reals each) for loads that expose
// contiguous rows (Load::kRaw).
template <typename T, int LR, bool PAD, int V>
__host__ __device__ constexpr int row_fwd_stage_bytes() {
    return row_rb_v<T>(LR, V) * (PAD ? LR : 2 * LR) * (int)sizeof(T);
}
template <typename T, int LR, bool PAD, int V, bool RAW>
__host__ __device__ constexpr bool row_fwd_staged() {
    return RAW && !PAD && (PAD ? LR : 2 * LR) % (16 / (int)sizeof(T)) == 0 &&
           (align16(row_smem_v<T>(LR, V)) + row_fwd_stage_bytes<T, LR, PAD, V>()) *
                   row_minb<T>(LR, V) <= kSmemPerSM;
}
template <typename T, int LR, bool PAD, int V, class Load>
__host__ __device__ constexpr int row_fwd_smem() {
    return row_fwd_staged<T, LR, PAD, V, Load::kRaw>()
               ? align16(row_smem_v<T>(LR, V)) + row_fwd_stage_bytes<T, LR, PAD, V>()
               : row_smem_v<T>(LR, V);
}
// Row inverse: staging of RB half-spectrum rows in the workspace's padded
// layout for tiled loads (Load::kTiled).
template <typename T, int LR, bool PAD, int V, bool TILED>
__host__ __device__ constexpr bool row_inv_staged() {
    return TILED && !PAD && (align16(row_smem_v<T>(LR, V)) + row_smem_v<T>(LR, V)) * row_minb<T>(LR, V) <=
                        kSmemPerSM;
}
template <typename T, int LR, bool PAD, int V, class Load>
__host__ __device__ constexpr int row_inv_smem() {
    return row_inv_staged<T, LR, PAD, V, Load::kTiled>()
               ? align16(row_smem_v<T>(LR, V)) + row_smem_v<T>(LR, V)
               : row_smem_v<T>(LR, V);
}
// Column: staging of one tile (its stored rows x CT columns, contiguous).
template <typename T, int LC, int NCM1, bool PAD, int V>
__host__ __device__ constexpr int col_stage_bytes() {
    return (PAD ? LC / 2 : LC) * col_ct_v<T>(LC, NCM1, V) * (int)sizeof(cplx<T>);
}
template <typename T, int LC, int NCM1, bool PAD, int V>
__host__ __device__ constexpr bool col_staged() {
    return !PAD && (align16(col_smem<T>(LC, col_ct_v<T>(LC, NCM1, V))) +
            col_stage_bytes<T, LC, NCM1, PAD, V>()) *
               col_minb<T>(LC, NCM1, V) <= kSmemPerSM;
}
// Unstaged column kernels take a second FFT workspace (ping-pong round
// trips, one barrier each instead of two) where it fits beside the CTAs per
// SM the variant asks for.
template <typename T, int LC, int NCM1, bool PAD, int V>
__host__ __device__ constexpr bool col_pp() {
    return !col_staged<T, LC, NCM1, PAD, V>() &&
           2 * align16(col_smem<T>(LC, col_ct_v<T>(LC, NCM1, V))) * col_minb<T>(LC, NCM1, V) <=
               kSmemPerSM;
}
template <typename T, int LC, int NCM1, bool PAD, int V>
__host__ __device__ constexpr int col_smem_total() {
    return col_staged<T, LC, NCM1, PAD, V>()
               ? align16(col_smem<T>(LC, col_ct_v<T>(LC, NCM1, V))) +
                     col_stage_bytes<T, LC, NCM1, PAD, V>()
           : col_pp<T, LC, NCM1, PAD, V>()
               ? 2 * align16(col_smem<T>(LC, col_ct_v<T>(LC, NCM1, V)))
               : col_smem<T>(LC, col_ct_v<T>(LC, NCM1, V));
}

// ---- full row groups of the tiled half spectrum ---------------------------------
// A full group (RB rows) moves its RB x ct tile chunks between shared memory
// and HBM with compile-time strides when the tile width ct is a power of two
// no larger than TT = LR / RPT (the threads of one row) and TT is a multiple
// of 16: thread tid owns chunk element e = tid % (RB ct) -- row rr = e / ct,
// column c = e % ct -- and the spectrum columns k = k0 + i TT, i < RPT, with
// k0 = (tid / (RB ct)) ct + c < TT, at HBM offsets (tid / (RB ct)) nrows ct
// + e + i TT nrows; column LR (tile LR / ct) belongs to the threads with
// tid < RB ct and c = 0.  f(std::integral_constant<int, CT>) runs the form;
// returns false (f not called) where the shape does not qualify.
template <int TT, class F>
__device__ __forceinline__ bool with_tile_width(int ct, F&& f) {
    if constexpr (TT % 16 != 0) {
        return false;
    } else {
        switch (ct) {
            case 1: f(std::integral_constant<int, 1>{}); return true;
            case 2: f(std::integral_constant<int, 2>{}); return true;
            case 4: f(std::integral_constant<int, 4>{}); return true;
            case 8: f(std::integral_constant<int, 8>{}); return true;
            case 16: f(std::integral_constant<int, 16>{}); return true;
            default: return false;
        }
    }
}

// ---- row forward ---------------------------------------------------------------
// Load:  cplx<T> operator()(int row, int n) -> z[n] = (x[2n], x[2n+1]);
//        static constexpr bool kRaw: true when x / pitch / bs expose plain
//        contiguous rows (then the kernel stages them with cp.async and
//        passes each staged pair through ld.fix())
// Store: void operator()(int row, int k, cplx<T> X), k in [0, LR]
//        static constexpr bool kTiled: true for the tiled half-spectrum store
//        (then the kernel writes whole tile chunks through base / nrows / ct /
//        bs itself); static constexpr bool kFinish: when true, every thread
//        calls finish(double* scratch) once, after a __syncthreads() at the end
// Dynamic shared memory: row_fwd_smem<T, LR, PAD, V, Load>().
template <typename T, int LR, bool PAD, int V, class Load, class Store>
__global__ void __launch_bounds__(row_threads<T>(LR, V), (row_fwd_minb<T, LR, PAD, V>()))
row_fwd_kernel(Load ld, Store st, int nrows, const cplx<T>* __restrict__ tw_lr,
               const cplx<T>* __restrict__ tw_2lr, const int* __restrict__ gate) {
    if (gate && gate[blockIdx.y * kGateStride]) return;
    constexpr int RPT = row_rpt<T>(LR, V);
    constexpr int TT = LR / RPT;
    constexpr int RB = row_rb_v<T>(LR, V);
    constexpr bool STAGED = row_fwd_staged<T, LR, PAD, V, Load::kRaw>();
    constexpr int NREAL = PAD ? LR : 2 * LR;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    T* stg = reinterpret_cast<T*>(smraw + align16(row_smem_v<T>(LR, V)));
    const int r = threadIdx.x / TT, t = threadIdx.x % TT;
    const int off = r * sm_len(LR + 1);
    const int ngroups = (nrows + RB - 1) / RB;
    auto issue = [&](int grp) {  // the group's rows -> stg (cp.async)
        if constexpr (STAGED) {
            constexpr int PER = 16 / (int)sizeof(T);
            constexpr int VPR = NREAL / PER;  // 16-byte vectors per row
            const int row0 = grp * RB;
            const int nr = nrows - row0 < RB ? nrows - row0 : RB;
            const T* src = ld.x + blockIdx.y * ld.bs + (size_t)row0 * ld.pitch;
            for (int f = threadIdx.x; f < nr * VPR; f += blockDim.x) {
                const int rr = f / VPR, e = (f - rr * VPR) * PER;
                cp_async16(stg + rr * NREAL + e, src + (size_t)rr * ld.pitch + e);
            }
            cp_async_commit();
        }
    };
    // split step of the real transform: X[k] = E + w^k O with
    // E = (Z[k] + conj Z[-k])/2, O = (Z[k] - conj Z[-k])/(2i), k in [0, LR]
    auto split_w = [&](cplx<T> zk, cplx<T> zn, cplx<T> w) {
        const cplx<T> A = mk<T>(zk.x + zn.x, zk.y - zn.y);
        const cplx<T> B = mk<T>(zk.x - zn.x, zk.y + zn.y);
        const cplx<T> O = mk<T>(B.y * T(0.5), -B.x * T(0.5));
        return cadd(cscale(A, T(0.5)), cmul(w, O));
    };
    auto split = [&](cplx<T> zk, cplx<T> zn, int k) {
        return split_w(zk, zn, __ldg(&tw_2lr[k]));
    };
    // transform of group grp from the strided registers v, and its store
    auto body = [&](int grp, cplx<T> (&v)[RPT]) {
        const int row = grp * RB + r;
        const bool valid = row < nrows;
        block_fft<T, LR, RPT, -1, 1, PAD>(v, t, sm, off, tw_lr);
#pragma unroll
        for (int m = 0; m < RPT; ++m) sm[smaddr_run<TT, 1 << 30>(t, m, 1, off)] = v[m];
        if (t == 0) sm[smaddr(LR, 1, off)] = v[0];  // Z[LR] = Z[0]: Z[-0] without a mask
        __syncthreads();
        if constexpr (Store::kTiled) {
            // each output reads Z[k] and Z[-k] from shared memory and goes
            // straight to its tile chunk (RB rows x ct columns, contiguous)
            const int row0 = grp * RB;
            const int nr = nrows - row0 < RB ? nrows - row0 : RB;
            const int ct = st.ct;
            cplx<T>* gbase = st.base + blockIdx.y * st.bs + (size_t)row0 * ct;
            auto store_full = [&](auto ctc) {
                constexpr int CT = decltype(ctc)::value;
                constexpr int CH = RB * CT;
                constexpr int ASTEP = TT + TT / 16;  // smaddr(k + TT) - smaddr(k)
                if constexpr (CT <= TT) {
                    const int tid = threadIdx.x, e = tid % CH, c = e % CT;
                    const int k0 = (tid / CH) * CT + c;
                    const int o = (e / CT) * sm_len(LR + 1);
                    const int ak = smaddr(k0, 1, o), an = smaddr(LR - k0, 1, o);
                    cplx<T>* dst = gbase + (size_t)(tid / CH) * st.nrows * CT + e;
                    const size_t jstep = (size_t)TT * st.nrows;
#pragma unroll
                    for (int i = 0; i < RPT; ++i)
                        dst[i * jstep] = split_w(sm[ak + i * ASTEP], sm[an - i * ASTEP],
                                                 __ldg(&tw_2lr[k0 + i * TT]));
                    if (tid < CH && c == 0) {  // k == LR: X = Re Z0 - Im Z0
                        const cplx<T> z0 = sm[ak];
                        gbase[(size_t)(LR / CT) * st.nrows * CT + e] = mk<T>(z0.x - z0.y, T(0));
                    }
                }
            };
            if (nr == RB && RB * TT == (int)blockDim.x && ct <= TT &&
                with_tile_width<TT>(ct, store_full))
                return;
            const int chunk = nr * ct;
            const int ntiles = LR / ct + 1;
            const int lct = __ffs(ct) - 1;  // ct is a power of two
            const bool full = nr == RB;
            const int lchunk = lct + ilog2c(RB);
            cplx<T>* base = st.base + blockIdx.y * st.bs + (size_t)row0 * ct;
            const int total = ntiles * chunk;
            // U outputs per thread at a time: their shared-memory reads and
            // twiddle loads are all issued before the first is used (U = 1
            // where the launch's register budget is below 96)
            constexpr int REGCAP = 65536 / (row_threads<T>(LR, V) * row_fwd_minb<T, LR, PAD, V>());
            constexpr int U = REGCAP < 96 ? 1 : (sizeof(T) == 4 ? 4 : 2);
            for (int f0 = threadIdx.x; f0 < total; f0 += U * blockDim.x) {
                cplx<T> zk[U], zn[U], w[U];
                size_t at[U];
                int kk[U];
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    const int f = f0 + u * (int)blockDim.x;
                    kk[u] = LR + 1;  // no output
                    if (f < total) {
                        const int j = full ? f >> lchunk : f / chunk, e = f - j * chunk;
                        const int rr = e >> lct, c = e & (ct - 1);
                        const int k = j * ct + c;
                        if (k <= LR) {
                            const int o = rr * sm_len(LR + 1);
                            kk[u] = k;
                            at[u] = (size_t)j * st.nrows * ct + e;
                            zk[u] = sm[smaddr(k & (LR - 1), 1, o)];
                            zn[u] = sm[smaddr((LR - k) & (LR - 1), 1, o)];
                            w[u] = __ldg(&tw_2lr[k < LR ? k : 0]);
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < U; ++u) {
                    if (kk[u] > LR) continue;
                    // k == LR: zk = Z[0], X = Re Z0 - Im Z0
                    const cplx<T> X = kk[u] == LR ? mk<T>(zk[u].x - zk[u].y, T(0))
                                                  : split_w(zk[u], zn[u], w[u]);
                    base[at[u]] = X;
                }
            }
        } else {
            const cplx<T> z0 = v[0];
#pragma unroll
            for (int m = 0; m < RPT; ++m) {
                const int k = t + m * TT;
                v[m] = split(v[m], sm[smaddr((LR - k) & (LR - 1), 1, off)], k);
            }
#pragma unroll
            for (int m = 0; m < RPT; ++m)
                if (valid) st(row, t + m * TT, v[m]);
            if (t == 0 && valid) st(row, LR, mk<T>(z0.x - z0.y, T(0)));
        }
    };
    if constexpr (STAGED) {
        // persistent loop: the next group's rows are staged during this one
        int grp = blockIdx.x;
        if (grp < ngroups) issue(grp);
        for (; grp < ngroups; grp += gridDim.x) {
            const bool valid = grp * RB + r < nrows;
            cplx<T> v[RPT];
            cp_async_wait_all();
            __syncthreads();
            const cplx<T>* srow = reinterpret_cast<const cplx<T>*>(stg + r * NREAL);
#pragma unroll
            for (int m = 0; m < RPT; ++m) {
                if (PAD && m >= RPT / 2) v[m] = mk<T>(0, 0);
                else v[m] = valid ? ld.fix(srow[t + m * TT]) : mk<T>(0, 0);
            }
            __syncthreads();
            if (grp + (int)gridDim.x < ngroups) issue(grp + gridDim.x);
            body(grp, v);
            __syncthreads();  // the workspace is rewritten by the next group
        }
    } else {
        // one group per CTA (a loop costs registers the unstaged kernel
        // cannot spare)
        const int grp = blockIdx.x;
        const int row = grp * RB + r;
        const bool valid = row < nrows;
        cplx<T> v[RPT];
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            if (PAD && m >= RPT / 2) v[m] = mk<T>(0, 0);
            else v[m] = valid ? ld(row, t + m * TT) : mk<T>(0, 0);
        }
        body(grp, v);
    }
    if constexpr (Store::kFinish) {
        __syncthreads();
        st.finish(reinterpret_cast<double*>(smraw));
    }
}

// ---- row inverse ----------------------------------------------------------------
// Load:  cplx<T> operator()(int row, int k), k in [0, LR]; kTiled as for the
//        forward store (whole tile chunks, staged with cp.async when the
//        staging buffer fits)
// Store: void operator()(int row, int n, cplx<T> z) -> (x[2n], x[2n+1]);
//        static constexpr bool kFinish (see row_fwd_kernel)
// Dynamic shared memory: row_inv_smem<T, LR, PAD, V, Load>().
template <typename T, int LR, bool PAD, int V, class Load, class Store>
__global__ void __launch_bounds__(row_threads<T>(LR, V), row_minb<T>(LR, V))
row_inv_kernel(Load ld, Store st, int nrows, const cplx<T>* __restrict__ tw_lr,
               const cplx<T>* __restrict__ tw_2lr, const int* __restrict__ gate) {
    if (gate && gate[blockIdx.y * kGateStride]) return;
    constexpr int RPT = row_rpt<T>(LR, V);
    constexpr int TT = LR / RPT;
    constexpr int RB = row_rb_v<T>(LR, V);
    constexpr bool STAGED = row_inv_staged<T, LR, PAD, V, Load::kTiled>();
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw + align16(row_smem_v<T>(LR, V)));
    const int r = threadIdx.x / TT, t = threadIdx.x % TT;
    const int off = r * sm_len(LR + 1);
    const int ngroups = (nrows + RB - 1) / RB;
    // the group's tile chunks (RB rows x ct columns, contiguous in HBM) into
    // `dst` in the padded row layout; cp.async when staged
    auto gather = [&](int grp, cplx<T>* dst) {
        if constexpr (Load::kTiled) {
            const int row0 = grp * RB;
            const int nr = nrows - row0 < RB ? nrows - row0 : RB;
            const int ct = ld.ct;
            const int chunk = nr * ct;
            const int ntiles = LR / ct + 1;
            const int lct = __ffs(ct) - 1;  // ct is a power of two
            const bool full = nr == RB;
            const int lchunk = lct + ilog2c(RB);
            const cplx<T>* base = ld.base + blockIdx.y * ld.bs + (size_t)row0 * ct;
            const int total = ntiles * chunk;
            auto fast = [&](auto ctc) {  // a full group: every load in flight at once
                constexpr int CT = decltype(ctc)::value;
                constexpr int CH = RB * CT;
                constexpr int ASTEP = TT + TT / 16;  // smaddr(k + TT) - smaddr(k)
                if constexpr (CT <= TT) {
                    const int tid = threadIdx.x, e = tid % CH, c = e % CT;
                    const int k0 = (tid / CH) * CT + c;
                    const int o = (e / CT) * sm_len(LR + 1);
                    const cplx<T>* src = base + (size_t)(tid / CH) * ld.nrows * CT + e;
                    const size_t jstep = (size_t)TT * ld.nrows;
                    const bool last = tid < CH && c == 0;  // column LR
                    cplx<T> val[RPT], vl;
#pragma unroll
                    for (int i = 0; i < RPT; ++i) val[i] = src[i * jstep];
                    if (last) vl = base[(size_t)(LR / CT) * ld.nrows * CT + e];
                    const int ak = smaddr(k0, 1, o);
#pragma unroll
                    for (int i = 0; i < RPT; ++i) dst[ak + i * ASTEP] = val[i];
                    if (last) dst[smaddr(LR, 1, o)] = vl;
                }
            };
            if (!STAGED && full && RB * TT == (int)blockDim.x && ct <= TT &&
                with_tile_width<TT>(ct, fast))
                return;
            if constexpr (STAGED) {
                for (int f = threadIdx.x; f < total; f += blockDim.x) {
                    const int j = full ? f >> lchunk : f / chunk, e = f - j * chunk;
                    const int rr = e >> lct, c = e & (ct - 1);
                    const int k = j * ct + c;
                    if (k > LR) continue;
                    cp_async_cplx<T>(&dst[smaddr(k, 1, rr * sm_len(LR + 1))],
                                     &base[(size_t)j * ld.nrows * ct + e]);
                }
                cp_async_commit();
            } else {
                // U loads in flight per thread before their stores: the
                // chunks come from L2 / HBM, and one dependent load at a time
                // left the kernel waiting on load latency
                constexpr int U = 8;
                for (int f0 = threadIdx.x; f0 < total; f0 += U * blockDim.x) {
                    cplx<T> val[U];
                    int at[U];
#pragma unroll
                    for (int u = 0; u < U; ++u) {
                        const int f = f0 + u * (int)blockDim.x;
                        at[u] = -1;
                        if (f < total) {
                            const int j = full ? f >> lchunk : f / chunk, e = f - j * chunk;
                            const int rr = e >> lct, c = e & (ct - 1);
                            const int k = j * ct + c;
                            if (k <= LR) {
                                at[u] = smaddr(k, 1, rr * sm_len(LR + 1));
                                val[u] = base[(size_t)j * ld.nrows * ct + e];
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < U; ++u)
                        if (at[u] >= 0) dst[at[u]] = val[u];
                }
            }
        }
    };
    // split step from `src` (padded rows), transform and store of group grp
    auto body = [&](int grp, const cplx<T>* src) {
        const int row = grp * RB + r;
        const bool valid = row < nrows;
        cplx<T> v[RPT];
        // padded-layout addresses of Z[k] and Z[LR - k]: per-thread bases
        // plus compile-time steps when TT is a multiple of 16
        constexpr int DSTEP = TT % 16 == 0 ? TT + TT / 16 : 0;
        const int ak = smaddr(t, 1, off), an = smaddr(LR - t, 1, off);
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            const int k = t + m * TT;
            const cplx<T> xk = src[DSTEP ? ak + m * DSTEP : smaddr(k, 1, off)];
            const cplx<T> xn = src[DSTEP ? an - m * DSTEP : smaddr(LR - k, 1, off)];
            const cplx<T> A = mk<T>(xk.x + xn.x, xk.y - xn.y);
            const cplx<T> B = mk<T>(xk.x - xn.x, xk.y + xn.y);
            const cplx<T> Bw = cmulc(B, __ldg(&tw_2lr[k]));  // B * exp(+2 pi i k / 2LR)
            v[m] = mk<T>(A.x - Bw.y, A.y + Bw.x);             // A + i Bw
        }
        __syncthreads();
        if constexpr (STAGED)
            if (grp + (int)gridDim.x < ngroups) gather(grp + gridDim.x, stg);
        block_fft<T, LR, RPT, +1, 1>(v, t, sm, off, tw_lr);
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            if (PAD && m >= RPT / 2) continue;
            if (valid) st(row, t + m * TT, v[m]);
        }
    };
    if constexpr (STAGED) {
        // persistent loop: the next group's chunks are staged during this one
        int grp = blockIdx.x;
        if (grp < ngroups) gather(grp, stg);
        for (; grp < ngroups; grp += gridDim.x) {
            cp_async_wait_all();
            __syncthreads();
            body(grp, stg);
            __syncthreads();  // the workspace is rewritten by the next group
        }
    } else {
        // one group per CTA
        const int grp = blockIdx.x;
        if constexpr (Load::kTiled) {
            gather(grp, sm);
        } else {
            const int row = grp * RB + r;
            const bool valid = row < nrows;
            for (int k = t; k <= LR; k += TT)
                sm[smaddr(k, 1, off)] = valid ? ld(row, k) : mk<T>(0, 0);
        }
        __syncthreads();
        body(grp, sm);
    }
    if constexpr (Store::kFinish) {
        __syncthreads();
        st.finish(reinterpret_cast<double*>(smraw));
    }
}

// ---- column forward * multiplier * inverse --------------------------------------
// Mult: cplx<T> operator()(cplx<T> X, int kx, int ky).  One unit = one tile
// of CT columns; instance blockIdx.y owns NCM1/CT + 1 contiguous tiles.
// Dynamic shared memory: col_smem_total<T, LC, NCM1, PAD, V>().
template <typename T, int LC, int NCM1, bool PAD, int V, class Mult>
__global__ void __launch_bounds__(col_threads<T>(LC, NCM1, V), col_minb<T>(LC, NCM1, V))
col_kernel(cplx<T>* __restrict__ spec, int nrows, Mult mul,
           const cplx<T>* __restrict__ tw_lc, const int* __restrict__ gate) {
    if (gate && gate[blockIdx.y * kGateStride]) return;
    constexpr int RPT = col_rpt<T>(LC, V);
    constexpr int CT = col_ct_v<T>(LC, NCM1, V);
    constexpr int TT = LC / RPT;
    constexpr int NTILES = NCM1 / CT + 1;
    constexpr bool STAGED = col_staged<T, LC, NCM1, PAD, V>();
    constexpr int ROWS = PAD ? LC / 2 : LC;  // stored rows of a tile
    // second workspace (elements from sm) of the ping-pong form, else 0
    constexpr int ALT = col_pp<T, LC, NCM1, PAD, V>()
                            ? align16(col_smem<T>(LC, CT)) / (int)sizeof(cplx<T>) : 0;
    constexpr int P1 = ALT ? ping_pong_next<LC, RPT>(0) : 0;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    cplx<T>* stg = reinterpret_cast<cplx<T>*>(smraw + align16(col_smem<T>(LC, CT)));
    const int c = threadIdx.x % CT, t = threadIdx.x / CT;
    cplx<T>* inst = spec + (size_t)blockIdx.y * NTILES * nrows * CT;
    auto issue = [&](int tile) {  // the tile's stored rows -> stg (cp.async)
        if constexpr (STAGED) {
            constexpr int NV = ROWS * CT * (int)sizeof(cplx<T>) / 16;
            const char* src = reinterpret_cast<const char*>(inst + (size_t)tile * nrows * CT);
            char* dst = reinterpret_cast<char*>(stg);
            for (int f = threadIdx.x; f < NV; f += blockDim.x) cp_async16(dst + 16 * f, src + 16 * f);
            cp_async_commit();
        }
    };
    // transform, multiply, inverse and store of tile `tile` from registers v
    auto body = [&](int tile, cplx<T> (&v)[RPT]) {
        cplx<T>* base = inst + (size_t)tile * nrows * CT;
        block_fft<T, LC, RPT, -1, CT, PAD, ALT>(v, t, sm, c, tw_lc);
        const int kx = tile * CT + c;
#pragma unroll
        for (int m = 0; m < RPT; ++m) v[m] = mul(v[m], kx, t + m * TT);
        block_fft<T, LC, RPT, +1, CT, false, ALT, P1>(v, t, sm, c, tw_lc);
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            if (PAD && m >= RPT / 2) continue;
            base[(size_t)(t + m * TT) * CT + c] = v[m];
        }
    };
    if constexpr (STAGED) {
        // persistent loop: the next tile is staged during this one
        int tile = blockIdx.x;
        if (tile < NTILES) issue(tile);
        for (; tile < NTILES; tile += gridDim.x) {
            cplx<T> v[RPT];
            cp_async_wait_all();
            __syncthreads();
#pragma unroll
            for (int m = 0; m < RPT; ++m) {
                if (PAD && m >= RPT / 2) v[m] = mk<T>(0, 0);
                else v[m] = stg[(t + m * TT) * CT + c];
            }
            __syncthreads();
            if (tile + (int)gridDim.x < NTILES) issue(tile + gridDim.x);
            body(tile, v);
            __syncthreads();  // the workspace is rewritten by the next tile
        }
    } else {
        // one tile per CTA (a loop costs registers the unstaged kernel cannot
        // spare)
        const int tile = blockIdx.x;
        const cplx<T>* base = inst + (size_t)tile * nrows * CT;
        cplx<T> v[RPT];
#pragma unroll
        for (int m = 0; m < RPT; ++m) {
            if (PAD && m >= RPT / 2) v[m] = mk<T>(0, 0);
            else v[m] = base[(size_t)(t + m * TT) * CT + c];
        }
        body(tile, v);
    }
}

// ---- split column (free space, the length-2LH column too long for one CTA) -------
// The zero-padded column transform of length M = 2 LH is evaluated as two
// length-LH halves.  With x[n] = 0 for n >= LH and w = exp(-2 pi i / M):
//   X[2m] = FFT_LH(x)[m],   X[2m+1] = FFT_LH(w^n x)[m],
// and for the kept outputs n < LH (unnormalised inverse, as col_kernel)
//   y[n] = IFFT_LH(K[2m] X[2m])[n] + w^-n IFFT_LH(K[2m+1] X[2m+1])[n].
// PARITY 0 writes its half to `acc` (a second spectrum-shaped buffer with the
// same tiled layout); PARITY 1 adds it and writes the column in place.  Each
// launch reads the untouched input column, so the two launches run back to
// back on one stream.  One column tile per CTA; shared memory col_smem<T>(LH, CT).
template <typename T, int LH, int NCM1, int V, int PARITY, class Mult>
__global__ void __launch_bounds__(col_threads<T>(LH, NCM1, V), col_minb<T>(LH, NCM1, V))
col_split_kernel(cplx<T>* __restrict__ spec, cplx<T>* __restrict__ acc, int nrows, Mult mul,
                 const cplx<T>* __restrict__ tw_lh, const cplx<T>* __restrict__ tw_m,
                 const int* __restrict__ gate) {
    if (gate && gate[blockIdx.y * kGateStride]) return;
    constexpr int RPT = col_rpt<T>(LH, V);
    constexpr int CT = col_ct_v<T>(LH, NCM1, V);
    constexpr int TT = LH / RPT;
    constexpr int NTILES = NCM1 / CT + 1;
    extern __shared__ __align__(16) unsigned char smraw[];
    cplx<T>* sm = reinterpret_cast<cplx<T>*>(smraw);
    const int c = threadIdx.x % CT, t = threadIdx.x / CT;
    const size_t off = (size_t)blockIdx.y * NTILES * nrows * CT + (size_t)blockIdx.x * nrows * CT;
    cplx<T>* base = spec + off;
    cplx<T>* abase = acc + off;
    cplx<T> v[RPT];
#pragma unroll
    for (int m = 0; m < RPT; ++m) {
        const int n = t + m * TT;
        v[m] = base[(size_t)n * CT + c];
        if constexpr (PARITY) v[m] = cmul(v[m], __ldg(&tw_m[n]));
    }
    block_fft<T, LH, RPT, -1, CT>(v, t, sm, c, tw_lh);
    const int kx = blockIdx.x * CT + c;
#pragma unroll
    for (int m = 0; m < RPT; ++m) v[m] = mul(v[m], kx, 2 * (t + m * TT) + PARITY);
    block_fft<T, LH, RPT, +1, CT>(v, t, sm, c, tw_lh);
#pragma unroll
    for (int m = 0; m < RPT; ++m) {
        const size_t i = (size_t)(t + m * TT) * CT + c;
        if constexpr (PARITY) {
            base[i] = cadd(cmulc(v[m], __ldg(&tw_m[t + m * TT])), abase[i]);
        } else {
            abase[i] = v[m];
        }
    }
}

}  // namespace asb
