// fft.cuh -- block-cooperative complex FFTs for sm_100a (FP64).
//
// One "team" of T = N/8 threads transforms one length-N sequence.  Thread t
// always holds the 8 elements at positions t + p*T (p = 0..7) in registers
// before the first pass and after the last pass, so a transform can start from
// values the thread loaded itself (coalesced: consecutive threads read
// consecutive elements) and its results can be consumed in place (pointwise
// products of several transforms need no shared-memory exchange).
//
// Algorithm: Stockham autosort, radix 8 while at least 8 remains, then one
// radix-4 or radix-2 pass (Govindaraju et al., "High performance discrete
// Fourier transforms on graphics processors", SC 2008).  Pass with stride Ns
// and radix R: butterfly j reads x[j + r*N/R], multiplies by
// W_N^{(j mod Ns) * r * N/(Ns*R)}, does a radix-R DFT and writes
// x'[(j div Ns)*Ns*R + (j mod Ns) + r*Ns].  Intermediate passes go through a
// per-team shared-memory buffer padded by one element every eight
// (pad(i) = i + i/8), which keeps the stride-8 writes of the first pass free of
// bank conflicts (one element every 16 for 8-byte elements).  Twiddles
// W_N^e = exp(-2 pi i e / N) are computed on the host in long double and stored
// in pass order (pass_twiddle_exponents): the twiddles of pass Ns, radix R sit
// at (Ns - 8) + (r - 1)*Ns + k, k = j mod Ns, so the lanes of a warp read
// consecutive entries instead of a gather with a stride of r*N/(Ns*R).
//
// DIR = -1: forward (unnormalised), DIR = +1: inverse (unnormalised).
// C = double2 (FP64) or float2 (FP32, the mixed-precision passes).
// All threads of the block must call the transform together: each pass ends in
// __syncthreads().
#pragma once
#include <cuda_runtime.h>

namespace ssg {

// ---- complex helpers for double2 (FP64) and float2 (FP32) -----------------
template <typename C> struct CT;
template <> struct CT<double2> {
    using R = double;
    __device__ __forceinline__ static double2 make(double x, double y) { return make_double2(x, y); }
};
template <> struct CT<float2> {
    using R = float;
    __device__ __forceinline__ static float2 make(float x, float y) { return make_float2(x, y); }
};

#define SSG_COMPLEX_OPS(C, R, MK)                                                                          \
    __device__ __forceinline__ C cadd(C a, C b) { return MK(a.x + b.x, a.y + b.y); }                        \
    __device__ __forceinline__ C csub(C a, C b) { return MK(a.x - b.x, a.y - b.y); }                        \
    __device__ __forceinline__ C cmul(C a, C b) { return MK(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x); } \
    __device__ __forceinline__ C cscale(C a, R s) { return MK(a.x * s, a.y * s); }                          \
    __device__ __forceinline__ C cconj(C a) { return MK(a.x, -a.y); }                                       \
    /* multiply by i*s (s real): (x + iy) * i s = -s y + i s x */                                          \
    __device__ __forceinline__ C cmul_is(C a, R s) { return MK(-s * a.y, s * a.x); }
SSG_COMPLEX_OPS(double2, double, make_double2)
SSG_COMPLEX_OPS(float2, float, make_float2)
#undef SSG_COMPLEX_OPS

// DIR * i * a
template <int DIR, typename C>
__device__ __forceinline__ C mul_i(C a) {
    return DIR < 0 ? CT<C>::make(a.y, -a.x) : CT<C>::make(-a.y, a.x);
}

template <int DIR, typename C>
__device__ __forceinline__ C twiddle(const C* __restrict__ tw, int e) {
    C w = __ldg(&tw[e]);
    return DIR < 0 ? w : CT<C>::make(w.x, -w.y);
}

// Host side: call emit(index, exponent) for every entry of the pass-ordered
// twiddle table of a length-N transform; table entry `index` must hold
// W_N^exponent.  The passes with stride Ns = 8, 64, ... and radix R take
// (R - 1)*Ns entries each, starting at Ns - 8 (the sizes telescope), so the
// table has N - 8 entries.
template <typename F>
inline void pass_twiddle_exponents(int N, F&& emit) {
    for (int ns = 8; ns < N; ns *= 8) {
        const int rem = N / ns, R = rem >= 8 ? 8 : rem, stride = N / (ns * R);
        for (int r = 1; r < R; ++r)
            for (int k = 0; k < ns; ++k) emit((ns - 8) + (r - 1) * ns + k, k * r * stride);
    }
}

// --- radix-R DFTs in registers ---------------------------------------------
template <int DIR, typename C>
__device__ __forceinline__ void dft2(C& a, C& b) {
    C t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR, typename C>
__device__ __forceinline__ void dft4(C& a0, C& a1, C& a2, C& a3) {
    C t0 = cadd(a0, a2), t1 = csub(a0, a2);
    C t2 = cadd(a1, a3), t3 = mul_i<DIR>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a1 = cadd(t1, t3);
    a2 = csub(t0, t2);
    a3 = csub(t1, t3);
}

template <int DIR, typename C>
__device__ __forceinline__ void dft8(C (&u)[8]) {
    using R = typename CT<C>::R;
    // even/odd split: E = DFT4(u0,u2,u4,u6), O = DFT4(u1,u3,u5,u7)
    C e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
    C o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    const R r = (R)0.70710678118654752440;  // 1/sqrt(2)
    // W8^1, W8^2, W8^3 with W8 = exp(DIR * 2 pi i / 8)
    C w1, w3;
    if (DIR < 0) {
        w1 = CT<C>::make(r * (o1.x + o1.y), r * (o1.y - o1.x));
        w3 = CT<C>::make(r * (o3.y - o3.x), -r * (o3.x + o3.y));
    } else {
        w1 = CT<C>::make(r * (o1.x - o1.y), r * (o1.x + o1.y));
        w3 = CT<C>::make(-r * (o3.x + o3.y), r * (o3.x - o3.y));
    }
    C w2 = mul_i<DIR>(o2);
    u[0] = cadd(e0, o0); u[4] = csub(e0, o0);
    u[1] = cadd(e1, w1); u[5] = csub(e1, w1);
    u[2] = cadd(e2, w2); u[6] = csub(e2, w2);
    u[3] = cadd(e3, w3); u[7] = csub(e3, w3);
}

template <int R, int DIR, typename C>
__device__ __forceinline__ void dft(C (&u)[R]) {
    if constexpr (R == 2) {
        dft2<DIR>(u[0], u[1]);
    } else if constexpr (R == 4) {
        dft4<DIR>(u[0], u[1], u[2], u[3]);
    } else {
        dft8<DIR>(u);
    }
}

// Shared-buffer padding: one spare element every 8 (16-byte elements) or every
// 16 (8-byte elements) keeps every pass's stores and loads free of bank
// conflicts for both element sizes.
template <typename C> __device__ __forceinline__ int fpad(int i);
template <> __device__ __forceinline__ int fpad<double2>(int i) { return i + (i >> 3); }
template <> __device__ __forceinline__ int fpad<float2>(int i) { return i + (i >> 4); }

template <int N>
struct FftShape {
    static constexpr int T = N / 8;            // threads per team
    static constexpr int BUF = N + N / 8;      // padded shared-memory elements per team
};

// butterflies of one pass, in registers
template <int N, int R, int NS, int DIR, typename C>
__device__ __forceinline__ void fft_butterflies(C (&v)[8], int t, const C* __restrict__ tw) {
    constexpr int Q = 8 / R;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = t + q * (N / 8);
        const int k = j & (NS - 1);
        C u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[q + r * Q];
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) u[r] = cmul(u[r], twiddle<DIR>(tw, (NS - 8) + (r - 1) * NS + k));
        }
        dft<R, DIR>(u);
#pragma unroll
        for (int r = 0; r < R; ++r) v[q + r * Q] = u[r];
    }
}

template <int N, int R, int NS, typename C>
__device__ __forceinline__ void fft_store(const C (&v)[8], int t, C* buf) {
    constexpr int Q = 8 / R;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = t + q * (N / 8);
        const int k = j & (NS - 1);
        const int idx = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[fpad<C>(idx + r * NS)] = v[q + r * Q];
    }
}

template <int N, typename C>
__device__ __forceinline__ void fft_load(C (&v)[8], int t, const C* buf) {
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = buf[fpad<C>(t + p * (N / 8))];
}

// Synchronisation between passes: the whole block, or only the team that owns
// the buffer (named barrier `id` over `n` threads, n a multiple of 32), which
// lets the teams of a block run independently.
struct BlockSync {
    __device__ __forceinline__ void operator()() const { __syncthreads(); }
};
struct TeamSync {
    int id, n;
    __device__ __forceinline__ void operator()() const {
        asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(n) : "memory");
    }
};

template <int N, int DIR, int NS, typename C, typename SYNC>
__device__ __forceinline__ void fft_stage(C (&v)[8], int t, C* buf, const C* __restrict__ tw, const SYNC& sync) {
    constexpr int REM = N / NS;
    constexpr int R = REM >= 8 ? 8 : REM;
    constexpr bool LAST = (NS * R == N);
    if constexpr (NS > 1) fft_load<N>(v, t, buf);
    fft_butterflies<N, R, NS, DIR>(v, t, tw);
    if constexpr (!LAST) {
        sync();
        fft_store<N, R, NS>(v, t, buf);
        sync();
        fft_stage<N, DIR, NS * R>(v, t, buf, tw, sync);
    }
}

// Length-N transform held by one team: v[p] = x[t + p*N/8] in, X[t + p*N/8] out.
template <int N, int DIR, typename C, typename SYNC = BlockSync>
__device__ __forceinline__ void fft_team(C (&v)[8], int t, C* buf, const C* __restrict__ tw,
                                         const SYNC& sync = SYNC{}) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two length >= 8");
    fft_stage<N, DIR, 1>(v, t, buf, tw, sync);
}

// K transforms of length N held by one team at once (v[s][p] = x_s[t + p*N/8]),
// pass by pass: each pass loads its twiddles once for the K transforms and
// synchronises once for all of them.  Per transform the operations are those
// of fft_team; the compiler may contract them into multiply-adds differently
// in the two forms, so results agree to rounding (measured: within a few ulps
// per transform), and each form reproduces itself bit for bit.  buf holds K
// padded buffers of FftShape<N>::BUF elements.
template <int N, int R, int NS, int DIR, int K, typename C>
__device__ __forceinline__ void fft_butterflies_k(C (&v)[K][8], int t, const C* __restrict__ tw) {
    constexpr int Q = 8 / R;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = t + q * (N / 8);
        const int k = j & (NS - 1);
        C w[R];
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) w[r] = twiddle<DIR>(tw, (NS - 8) + (r - 1) * NS + k);
        }
#pragma unroll
        for (int s = 0; s < K; ++s) {
            C u[R];
#pragma unroll
            for (int r = 0; r < R; ++r) u[r] = v[s][q + r * Q];
            if constexpr (NS > 1) {
#pragma unroll
                for (int r = 1; r < R; ++r) u[r] = cmul(u[r], w[r]);
            }
            dft<R, DIR>(u);
#pragma unroll
            for (int r = 0; r < R; ++r) v[s][q + r * Q] = u[r];
        }
    }
}

template <int N, int DIR, int NS, int K, typename C, typename SYNC>
__device__ __forceinline__ void fft_stage_k(C (&v)[K][8], int t, C* buf, const C* __restrict__ tw, const SYNC& sync) {
    constexpr int REM = N / NS;
    constexpr int R = REM >= 8 ? 8 : REM;
    constexpr bool LAST = (NS * R == N);
    if constexpr (NS > 1) {
#pragma unroll
        for (int s = 0; s < K; ++s) fft_load<N>(v[s], t, buf + s * FftShape<N>::BUF);
    }
    fft_butterflies_k<N, R, NS, DIR, K>(v, t, tw);
    if constexpr (!LAST) {
        sync();
#pragma unroll
        for (int s = 0; s < K; ++s) fft_store<N, R, NS>(v[s], t, buf + s * FftShape<N>::BUF);
        sync();
        fft_stage_k<N, DIR, NS * R, K>(v, t, buf, tw, sync);
    }
}

template <int N, int DIR, int K, typename C, typename SYNC = BlockSync>
__device__ __forceinline__ void fft_team_k(C (&v)[K][8], int t, C* buf, const C* __restrict__ tw,
                                           const SYNC& sync = SYNC{}) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two length >= 8");
    fft_stage_k<N, DIR, 1, K>(v, t, buf, tw, sync);
}

}  // namespace ssg
