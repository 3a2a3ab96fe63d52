// Register-resident Stockham FFT for one CTA-cooperative transform.
//
// A length-L complex transform is carried by L/RPT threads, each holding RPT
// elements in registers.  Thread t always holds elements t + m*(L/RPT),
// m = 0..RPT-1 (the "strided pattern") before and after the transform, and
// the output is in natural order.  The transform is the Stockham autosort
// formulation (Govindaraju et al., "High performance discrete Fourier
// transforms on graphics processors", SC'08): stage s with radix R and span
// Ns reads x[j + r L/R], twiddles input r by w_{Ns R}^{r (j mod Ns)}, does a
// radix-R DFT and writes y[(j div Ns) Ns R + (j mod Ns) + r Ns].  Each thread
// runs RPT/R butterflies per stage (j = t + q L/RPT), whose inputs are exactly
// its own strided registers, so only the stage outputs go through shared
// memory; the last stage's outputs land back in the strided pattern and stay
// in registers.  Stages are radix 16 (the remainder last), so a 4096-point
// transform makes two shared-memory round trips.
//
// Shared memory is addressed as (i + i/16) * S + off: the 1-in-16 padding
// breaks the power-of-two strides of the stage writes, S > 1 interleaves S
// independent transforms element by element (the column kernels).
#pragma once

#include "common.cuh"

namespace asb {

// cos/sin(2 pi k / 16), k = 0..7, as plain mathematical constants.
template <typename T>
__device__ __forceinline__ void unit16(int k, T& c, T& s) {
    const T c1 = T(0.92387953251128675613), s1 = T(0.38268343236508977173);
    const T h = T(0.70710678118654752440);
    switch (k) {
        case 0: c = T(1); s = T(0); break;
        case 1: c = c1; s = s1; break;
        case 2: c = h; s = h; break;
        case 3: c = s1; s = c1; break;
        case 4: c = T(0); s = T(1); break;
        case 5: c = -s1; s = c1; break;
        case 6: c = -h; s = h; break;
        default: c = -c1; s = s1; break;
    }
}

// a * exp(DIR * 2 pi i k / R) for a compile-time R in {2,4,8,16}.
template <int R, int DIR, typename T>
__device__ __forceinline__ cplx<T> rot_const(cplx<T> a, int k) {
    const int k16 = k * (16 / R);
    if (k16 == 0) return a;
    if (k16 == 4) return mul_i<DIR>(a);
    T c, s;
    unit16<T>(k16, c, s);
    const T sn = DIR < 0 ? -s : s;
    return mk<T>(a.x * c - a.y * sn, a.x * sn + a.y * c);
}

// cos and tan of 2 pi k / 16, k in {1, 2, 3, 5, 6, 7}, as plain
// mathematical constants (tan(pi/8) = sqrt(2) - 1, tan(3 pi/8) = sqrt(2) + 1)
template <typename T>
__device__ __forceinline__ void unit16_cos_tan(int k, T& c, T& t) {
    const T c1 = T(0.92387953251128675613), s1 = T(0.38268343236508977173);
    const T h = T(0.70710678118654752440);
    const T t1 = T(0.41421356237309504880), t3 = T(2.41421356237309504880);
    switch (k) {
        case 1: c = c1; t = t1; break;
        case 2: c = h; t = T(1); break;
        case 3: c = s1; t = t3; break;
        case 5: c = -s1; t = -t3; break;
        case 6: c = -h; t = T(-1); break;
        default: c = -c1; t = -t1; break;
    }
}

// The radix-2 butterfly with the odd input rotated by exp(DIR 2 pi i k / R):
// lo = e + w o, hi = e - w o.  A general rotation is factored as
// w o = c (o.x - t o.y, o.y + t o.x), t = tan of the angle (cos c != 0), and
// the factor c is folded into the two outputs' fused multiply-adds: six
// instructions instead of a four-instruction rotation and four additions.
template <int R, int DIR, typename T>
__device__ __forceinline__ void bfly_rot(cplx<T> e, cplx<T> o, int k, cplx<T>& lo, cplx<T>& hi) {
    const int k16 = k * (16 / R);
    if (k16 == 0) {
        lo = cadd(e, o);
        hi = csub(e, o);
    } else if (k16 == 4) {
        const cplx<T> w = mul_i<DIR>(o);
        lo = cadd(e, w);
        hi = csub(e, w);
    } else {
        T c, t;
        unit16_cos_tan<T>(k16, c, t);
        if (DIR < 0) t = -t;
        const T ux = fma(-t, o.y, o.x), uy = fma(t, o.x, o.y);
        lo = mk<T>(fma(c, ux, e.x), fma(c, uy, e.y));
        hi = mk<T>(fma(-c, ux, e.x), fma(-c, uy, e.y));
    }
}

// In-register DFT of R points (natural order in and out), radix-2 DIT split.
template <int R, int DIR, typename T>
__device__ __forceinline__ void dft(cplx<T>* a) {
    if constexpr (R == 1) {
        return;
    } else if constexpr (R == 2) {
        const cplx<T> t = a[0];
        a[0] = cadd(t, a[1]);
        a[1] = csub(t, a[1]);
    } else if constexpr (R == 4) {
        const cplx<T> s02 = cadd(a[0], a[2]), d02 = csub(a[0], a[2]);
        const cplx<T> s13 = cadd(a[1], a[3]);
        const cplx<T> d13 = mul_i<DIR>(csub(a[1], a[3]));
        a[0] = cadd(s02, s13);
        a[2] = csub(s02, s13);
        a[1] = cadd(d02, d13);
        a[3] = csub(d02, d13);
    } else {
        cplx<T> e[R / 2], o[R / 2];
#pragma unroll
        for (int i = 0; i < R / 2; ++i) { e[i] = a[2 * i]; o[i] = a[2 * i + 1]; }
        dft<R / 2, DIR, T>(e);
        dft<R / 2, DIR, T>(o);
#pragma unroll
        for (int k = 0; k < R / 2; ++k) bfly_rot<R, DIR, T>(e[k], o[k], k, a[k], a[k + R / 2]);
    }
}

// The DFT of R points whose upper half a[R/2 .. R-1] is zero (the first
// stage of a zero-padded transform): with w = exp(DIR 2 pi i / R),
//   X[2k] = DFT_{R/2}(a)[k],   X[2k+1] = DFT_{R/2}(a[n] w^n)[k],  n < R/2,
// two half-length DFTs instead of the full one on zeros (x + 0 is not folded
// by the compiler: -0 + 0 = +0).
template <int R, int DIR, typename T>
__device__ __forceinline__ void dft_upper_zero(cplx<T>* a) {
    cplx<T> b[R / 2], c[R / 2];
#pragma unroll
    for (int n = 0; n < R / 2; ++n) {
        b[n] = a[n];
        c[n] = rot_const<R, DIR, T>(a[n], n);
    }
    dft<R / 2, DIR, T>(b);
    dft<R / 2, DIR, T>(c);
#pragma unroll
    for (int k = 0; k < R / 2; ++k) {
        a[2 * k] = b[k];
        a[2 * k + 1] = c[k];
    }
}

__host__ __device__ constexpr int ilog2c(int v) { return v <= 1 ? 0 : 1 + ilog2c(v >> 1); }

// Radix of stage `s` for a length-L transform with at most RMAX per stage.
__host__ __device__ constexpr int stage_radix(int L, int RMAX, int s) {
    int rem = L;
    for (int i = 0; i < s; ++i) rem /= (rem >= RMAX ? RMAX : rem);
    return rem >= RMAX ? RMAX : rem;
}
__host__ __device__ constexpr int num_stages(int L, int RMAX) {
    int n = 0, rem = L;
    while (rem > 1) { rem /= (rem >= RMAX ? RMAX : rem); ++n; }
    return n;
}

__device__ __forceinline__ int smaddr(int i, int S, int off) { return (i + (i >> 4)) * S + off; }

// smaddr(i0 + m * STEP) as a per-thread base plus a compile-time offset where
// the padding term splits.  For STEP a multiple of 16, (i0 + m STEP) >> 4 =
// (i0 >> 4) + m STEP / 16.  RUN is the length (a power of two) of the
// RUN-aligned group that every i0 + m STEP stays in; for RUN <= 16 that group
// lies inside one 16-element block, so the padding term does not change
// with m.
template <int STEP, int RUN>
__device__ __forceinline__ int smaddr_run(int i0, int m, int S, int off) {
    if constexpr (STEP % 16 == 0) return smaddr(i0, S, off) + m * (STEP + STEP / 16) * S;
    else if constexpr (RUN <= 16) return smaddr(i0, S, off) + m * STEP * S;
    else return smaddr(i0 + m * STEP, S, off);
}

// a * w (forward) or a * conj(w) (inverse), w from the exp(-2 pi i k/L) table
template <int DIR, typename V>
__device__ __forceinline__ V tw_apply(V a, V w) {
    return DIR < 0 ? cmul(a, w) : cmulc(a, w);
}

// Shared-memory elements needed by one transform of length L (padded).
__host__ __device__ constexpr int sm_len(int L) { return L + L / 16 + 1; }

template <typename T, int L, int RPT, int DIR, int S, int STAGE, int SPAN, bool HZ, int ALT,
          int P0>
__device__ __forceinline__ void fft_stages(cplx<T> (&v)[RPT], int t, cplx<T>* sm, int off,
                                           const cplx<T>* __restrict__ tw) {
    constexpr int RMAX = RPT < 16 ? RPT : 16;
    constexpr int NST = num_stages(L, RMAX);
    if constexpr (STAGE < NST) {
        constexpr int R = stage_radix(L, RMAX, STAGE);
        constexpr int TT = L / RPT;   // threads per transform
        constexpr int Q = RPT / R;    // butterflies per thread
        constexpr bool LAST = (STAGE == NST - 1);
        static_assert(RPT % R == 0, "radix must divide RPT");
        // this round trip's workspace: with ALT > 0, round trips alternate
        // between sm and sm + ALT, starting at parity P0
        cplx<T>* ws = (ALT > 0 && ((STAGE + P0) & 1)) ? sm + ALT : sm;
#pragma unroll
        for (int q = 0; q < Q; ++q) {
            const int j = t + q * TT;
            cplx<T> a[R];
#pragma unroll
            for (int r = 0; r < R; ++r) a[r] = v[q + r * Q];
            if constexpr (SPAN > 1) {
                // w^r for r = 1..R-1 from the loaded powers w, w^2, w^4, w^8
                // (products at most three deep), applied as each is formed.
                // w^(2^e) = exp(-2 pi i jm / (SPAN R / 2^e)) is entry jm of the
                // length-(SPAN R / 2^e) table, so consecutive threads (jm)
                // read consecutive entries instead of a stride of L/(SPAN R).
                const int jm = j % SPAN;
                const cplx<T>* __restrict__ tb = tw - L;  // tables at offset = length
                const cplx<T> w1 = __ldg(&tb[SPAN * R + jm]);
                a[1] = tw_apply<DIR>(a[1], w1);
                if constexpr (R >= 4) {
                    const cplx<T> w2 = __ldg(&tb[SPAN * R / 2 + jm]);
                    a[2] = tw_apply<DIR>(a[2], w2);
                    const cplx<T> w3 = cmul(w2, w1);
                    a[3] = tw_apply<DIR>(a[3], w3);
                    if constexpr (R >= 8) {
                        const cplx<T> w4 = __ldg(&tb[SPAN * R / 4 + jm]);
                        a[4] = tw_apply<DIR>(a[4], w4);
                        a[5] = tw_apply<DIR>(a[5], cmul(w4, w1));
                        a[6] = tw_apply<DIR>(a[6], cmul(w4, w2));
                        a[7] = tw_apply<DIR>(a[7], cmul(w4, w3));
                        if constexpr (R >= 16) {
                            const cplx<T> w8 = __ldg(&tb[SPAN * R / 8 + jm]);
                            a[8] = tw_apply<DIR>(a[8], w8);
                            a[9] = tw_apply<DIR>(a[9], cmul(w8, w1));
                            a[10] = tw_apply<DIR>(a[10], cmul(w8, w2));
                            a[11] = tw_apply<DIR>(a[11], cmul(w8, w3));
                            const cplx<T> w12 = cmul(w8, w4);
                            a[12] = tw_apply<DIR>(a[12], w12);
                            a[13] = tw_apply<DIR>(a[13], cmul(w12, w1));
                            a[14] = tw_apply<DIR>(a[14], cmul(w12, w2));
                            a[15] = tw_apply<DIR>(a[15], cmul(w12, w3));
                        }
                    }
                }
            }
            // the zero upper half of the input (HZ) is the upper half of
            // every first-stage butterfly: a[r] = v[q + r Q] with v[m] = 0
            // for m >= RPT / 2 exactly when r >= R / 2
            if constexpr (HZ && STAGE == 0 && R >= 2)
                dft_upper_zero<R, DIR, T>(a);
            else
                dft<R, DIR, T>(a);
            if constexpr (LAST) {
#pragma unroll
                for (int r = 0; r < R; ++r) v[q + r * Q] = a[r];
            } else {
                const int base = (j / SPAN) * SPAN * R + (j % SPAN);
#pragma unroll
                for (int r = 0; r < R; ++r) ws[smaddr_run<SPAN, SPAN * R>(base, r, S, off)] = a[r];
            }
        }
        if constexpr (!LAST) {
            __syncthreads();
#pragma unroll
            for (int m = 0; m < RPT; ++m) v[m] = ws[smaddr_run<TT, 1 << 30>(t, m, S, off)];
            // one workspace: nobody writes it again before everyone has read
            // it.  Two (ALT > 0): the next round trip writes the other one,
            // and the one after that follows the next round trip's barrier,
            // which every thread reaches only after this read.
            if constexpr (ALT == 0) __syncthreads();
            fft_stages<T, L, RPT, DIR, S, STAGE + 1, SPAN * R, HZ, ALT, P0>(v, t, sm, off, tw);
        }
    }
}

// Length-L transform of the strided register pattern; DIR = -1 forward
// (exp(-2 pi i jk/L)), +1 inverse, both unnormalised.  tw points at the
// length-L table exp(-2 pi i k / L), k < L, inside one array that holds the
// table of every power-of-two length M <= L at offset M (so tw - L is the
// array base and the stages read the shorter tables).  Every thread of the CTA must
// call this (it contains __syncthreads), including threads whose transform
// is a dummy.  HZ: the upper half of the input is zero (v[m] = 0 for
// m >= RPT / 2, a zero-padded transform); its first stage skips the zeros.
// ALT > 0: a second workspace of the same shape at sm + ALT (elements); the
// shared-memory round trips alternate between the two, which saves the
// barrier after each read.  The first round trip uses parity P0 (0: sm,
// 1: sm + ALT); a caller that runs two transforms back to back without a
// barrier between them starts the second at ping_pong_next<L, RPT>(P0), the
// workspace the first one did not read last.
template <typename T, int L, int RPT, int DIR, int S, bool HZ = false, int ALT = 0, int P0 = 0>
__device__ __forceinline__ void block_fft(cplx<T> (&v)[RPT], int t, cplx<T>* sm, int off,
                                          const cplx<T>* __restrict__ tw) {
    static_assert(L % RPT == 0, "L must be a multiple of RPT");
    fft_stages<T, L, RPT, DIR, S, 0, 1, HZ, ALT, P0>(v, t, sm, off, tw);
}

// parity of the first round trip after a ping-pong transform that started at
// P0: the workspace its last round trip did not read
template <int L, int RPT>
__host__ __device__ constexpr int ping_pong_next(int p0) {
    return (p0 + num_stages(L, RPT < 16 ? RPT : 16) - 1) & 1;
}

}  // namespace asb
