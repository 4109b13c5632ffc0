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
// bank conflicts.  Twiddles come from a table W_N^e = exp(-2 pi i e / N)
// computed on the host in long double.
//
// DIR = -1: forward (unnormalised), DIR = +1: inverse (unnormalised).
// All threads of the block must call the transform together: each pass ends in
// __syncthreads().
#pragma once
#include <cuda_runtime.h>

namespace ssg {

__device__ __forceinline__ double2 cadd(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 csub(double2 a, double2 b) { return make_double2(a.x - b.x, a.y - b.y); }
__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cscale(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
// multiply by i*s (s real): (x + iy) * i s = -s y + i s x
__device__ __forceinline__ double2 cmul_is(double2 a, double s) { return make_double2(-s * a.y, s * a.x); }

// DIR * i * a
template <int DIR>
__device__ __forceinline__ double2 mul_i(double2 a) {
    return DIR < 0 ? make_double2(a.y, -a.x) : make_double2(-a.y, a.x);
}

template <int DIR>
__device__ __forceinline__ double2 twiddle(const double2* __restrict__ tw, int e) {
    double2 w = __ldg(&tw[e]);
    return DIR < 0 ? w : make_double2(w.x, -w.y);
}

// --- radix-R DFTs in registers ---------------------------------------------
template <int DIR>
__device__ __forceinline__ void dft2(double2& a, double2& b) {
    double2 t = a;
    a = cadd(t, b);
    b = csub(t, b);
}

template <int DIR>
__device__ __forceinline__ void dft4(double2& a0, double2& a1, double2& a2, double2& a3) {
    double2 t0 = cadd(a0, a2), t1 = csub(a0, a2);
    double2 t2 = cadd(a1, a3), t3 = mul_i<DIR>(csub(a1, a3));
    a0 = cadd(t0, t2);
    a1 = cadd(t1, t3);
    a2 = csub(t0, t2);
    a3 = csub(t1, t3);
}

template <int DIR>
__device__ __forceinline__ void dft8(double2 (&u)[8]) {
    // even/odd split: E = DFT4(u0,u2,u4,u6), O = DFT4(u1,u3,u5,u7)
    double2 e0 = u[0], e1 = u[2], e2 = u[4], e3 = u[6];
    double2 o0 = u[1], o1 = u[3], o2 = u[5], o3 = u[7];
    dft4<DIR>(e0, e1, e2, e3);
    dft4<DIR>(o0, o1, o2, o3);
    const double r = 0.70710678118654752440;  // 1/sqrt(2)
    // W8^1, W8^2, W8^3 with W8 = exp(DIR * 2 pi i / 8)
    double2 w1, w3;
    if (DIR < 0) {
        w1 = make_double2(r * (o1.x + o1.y), r * (o1.y - o1.x));
        w3 = make_double2(r * (o3.y - o3.x), -r * (o3.x + o3.y));
    } else {
        w1 = make_double2(r * (o1.x - o1.y), r * (o1.x + o1.y));
        w3 = make_double2(-r * (o3.x + o3.y), r * (o3.x - o3.y));
    }
    double2 w2 = mul_i<DIR>(o2);
    u[0] = cadd(e0, o0); u[4] = csub(e0, o0);
    u[1] = cadd(e1, w1); u[5] = csub(e1, w1);
    u[2] = cadd(e2, w2); u[6] = csub(e2, w2);
    u[3] = cadd(e3, w3); u[7] = csub(e3, w3);
}

template <int R, int DIR>
__device__ __forceinline__ void dft(double2 (&u)[R]) {
    if constexpr (R == 2) {
        dft2<DIR>(u[0], u[1]);
    } else if constexpr (R == 4) {
        dft4<DIR>(u[0], u[1], u[2], u[3]);
    } else {
        dft8<DIR>(u);
    }
}

__device__ __forceinline__ int fpad(int i) { return i + (i >> 3); }

template <int N>
struct FftShape {
    static constexpr int T = N / 8;            // threads per team
    static constexpr int BUF = N + N / 8;      // padded shared-memory elements per team
};

// butterflies of one pass, in registers
template <int N, int R, int NS, int DIR>
__device__ __forceinline__ void fft_butterflies(double2 (&v)[8], int t, const double2* __restrict__ tw) {
    constexpr int Q = 8 / R;
    constexpr int STRIDE = N / (NS * R);
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = t + q * (N / 8);
        const int k = j & (NS - 1);
        double2 u[R];
#pragma unroll
        for (int r = 0; r < R; ++r) u[r] = v[q + r * Q];
        if constexpr (NS > 1) {
#pragma unroll
            for (int r = 1; r < R; ++r) u[r] = cmul(u[r], twiddle<DIR>(tw, k * r * STRIDE));
        }
        dft<R, DIR>(u);
#pragma unroll
        for (int r = 0; r < R; ++r) v[q + r * Q] = u[r];
    }
}

template <int N, int R, int NS>
__device__ __forceinline__ void fft_store(const double2 (&v)[8], int t, double2* buf) {
    constexpr int Q = 8 / R;
#pragma unroll
    for (int q = 0; q < Q; ++q) {
        const int j = t + q * (N / 8);
        const int k = j & (NS - 1);
        const int idx = (j - k) * R + k;
#pragma unroll
        for (int r = 0; r < R; ++r) buf[fpad(idx + r * NS)] = v[q + r * Q];
    }
}

template <int N>
__device__ __forceinline__ void fft_load(double2 (&v)[8], int t, const double2* buf) {
#pragma unroll
    for (int p = 0; p < 8; ++p) v[p] = buf[fpad(t + p * (N / 8))];
}

template <int N, int DIR, int NS>
__device__ __forceinline__ void fft_stage(double2 (&v)[8], int t, double2* buf, const double2* __restrict__ tw) {
    constexpr int REM = N / NS;
    constexpr int R = REM >= 8 ? 8 : REM;
    constexpr bool LAST = (NS * R == N);
    if constexpr (NS > 1) fft_load<N>(v, t, buf);
    fft_butterflies<N, R, NS, DIR>(v, t, tw);
    if constexpr (!LAST) {
        __syncthreads();
        fft_store<N, R, NS>(v, t, buf);
        __syncthreads();
        fft_stage<N, DIR, NS * R>(v, t, buf, tw);
    }
}

// Length-N transform held by one team: v[p] = x[t + p*N/8] in, X[t + p*N/8] out.
template <int N, int DIR>
__device__ __forceinline__ void fft_team(double2 (&v)[8], int t, double2* buf, const double2* __restrict__ tw) {
    static_assert(N >= 8 && (N & (N - 1)) == 0, "power-of-two length >= 8");
    fft_stage<N, DIR, 1>(v, t, buf, tw);
}

}  // namespace ssg
