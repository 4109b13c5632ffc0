// fft_warp.cuh -- length-1024 complex FFT held by one warp (sm_100a).
//
// Four-step factorisation N = 32 x 32 (Bailey, "FFTs in external or
// hierarchical memory", J. Supercomputing 4, 1990): with n = n1 + 32 n2 and
// k = k1 + 32 k2,
//   X[k1 + 32 k2] = sum_n1 W32^(n1 k2) W1024^(n1 k1) sum_n2 x[n1 + 32 n2] W32^(n2 k1).
// Lane n1 holds x[n1 + 32 q], q = 0..31, in registers; it transforms over q
// (a 32-point DFT in registers), multiplies by W1024^(n1 k1), and the warp
// transposes once through a 32 x 33 buffer (row padding keeps both the
// row-wise stores and the column-wise loads free of bank conflicts), after
// which lane k1 transforms over n1 and holds X[k1 + 32 k2] in register k2:
// natural order, the same layout as the input.  One exchange per transform,
// synchronised by __syncwarp only, against three block-wide exchanges for the
// radix-8 team transform of fft.cuh.
//
// DIR = -1 forward (unnormalised), +1 inverse (unnormalised).  C = double2 or
// float2.  The twiddles W1024^(n1 k1) come from a table laid out
// [k1][n1] (warp_twiddle_exponents), so lanes read consecutive entries; the
// 32-point twiddles are the exact values cos(k pi/16), written as constants.
#pragma once
#include "fft.cuh"

namespace ssg {

// cos(k pi / 16), k = 0..8, correctly rounded (nested radicals:
// cos(pi/8) = sqrt(2 + sqrt 2)/2, cos(pi/16) = sqrt(2 + sqrt(2 + sqrt 2))/2, ...)
template <typename R> __device__ __forceinline__ R cos16(int k);
template <> __device__ __forceinline__ double cos16<double>(int k) {
    switch (k) {
        case 0: return 1.0;
        case 1: return 0.9807852804032304;
        case 2: return 0.9238795325112867;
        case 3: return 0.8314696123025452;
        case 4: return 0.7071067811865476;
        case 5: return 0.5555702330196022;
        case 6: return 0.3826834323650898;
        case 7: return 0.19509032201612828;
        default: return 0.0;
    }
}
template <> __device__ __forceinline__ float cos16<float>(int k) {
    switch (k) {
        case 0: return 1.0f;
        case 1: return 0.9807852506637573f;
        case 2: return 0.9238795042037964f;
        case 3: return 0.8314695954322815f;
        case 4: return 0.7071067690849304f;
        case 5: return 0.5555702447891235f;
        case 6: return 0.3826834261417389f;
        case 7: return 0.19509032368659973f;
        default: return 0.0f;
    }
}

// a * W32^e with W32 = exp(DIR 2 pi i / 32), 0 <= e < 16 (a compile-time
// constant once the callers' loops are unrolled: the branches fold)
template <int DIR, typename C>
__device__ __forceinline__ C mul_w32(C a, int e) {
    using R = typename CT<C>::R;
    if (e == 0) return a;
    if (e == 8) return mul_i<DIR>(a);
    // cos(2 pi e/32) and sin(2 pi e/32) for 0 < e < 16
    const R c = e < 8 ? cos16<R>(e) : -cos16<R>(16 - e);
    const R s = e < 8 ? cos16<R>(8 - e) : cos16<R>(e - 8);
    const R si = DIR < 0 ? -s : s;
    return CT<C>::make(a.x * c - a.y * si, a.x * si + a.y * c);
}

__device__ __forceinline__ constexpr int brev5(int k) {
    return ((k & 1) << 4) | ((k & 2) << 2) | (k & 4) | ((k & 8) >> 2) | ((k & 16) >> 4);
}

// 32-point DFT of u in registers: radix-2 decimation in frequency, then the
// bit-reversal permutation (a renaming of registers).
template <int DIR, typename C>
__device__ __forceinline__ void dft32(C (&u)[32]) {
#pragma unroll
    for (int s = 16; s >= 1; s >>= 1) {
#pragma unroll
        for (int b = 0; b < 32; b += 2 * s) {
#pragma unroll
            for (int j = 0; j < s; ++j) {
                const C a = u[b + j], c = u[b + j + s];
                u[b + j] = cadd(a, c);
                u[b + j + s] = mul_w32<DIR>(csub(a, c), j * (16 / s));
            }
        }
    }
    C t[32];
#pragma unroll
    for (int k = 0; k < 32; ++k) t[k] = u[brev5(k)];
#pragma unroll
    for (int k = 0; k < 32; ++k) u[k] = t[k];
}

// Elements of the warp exchange buffer: 32 rows of 33.
constexpr int kWarpFftBuf = 32 * 33;

// Length-1024 transform held by one warp: v[q] = x[lane + 32 q] in,
// X[lane + 32 q] out.  buf (kWarpFftBuf elements) is private to the warp;
// the call begins with __syncwarp, so the warp's earlier reads of buf are done.
// SMEM_TW: tw points to a copy of the table in shared memory (read with
// plain loads instead of through the read-only data cache).
template <int DIR, typename C, bool SMEM_TW = false>
__device__ __forceinline__ void fft_warp1024(C (&v)[32], int lane, C* buf, const C* __restrict__ tw) {
    dft32<DIR>(v);
#pragma unroll
    for (int k1 = 1; k1 < 32; ++k1) {
        C w;
        if constexpr (SMEM_TW) {
            w = tw[k1 * 32 + lane];
            if (DIR > 0) w = CT<C>::make(w.x, -w.y);
        } else {
            w = twiddle<DIR>(tw, k1 * 32 + lane);
        }
        v[k1] = cmul(v[k1], w);
    }
    __syncwarp();
#pragma unroll
    for (int k1 = 0; k1 < 32; ++k1) buf[k1 * 33 + lane] = v[k1];
    __syncwarp();
#pragma unroll
    for (int n1 = 0; n1 < 32; ++n1) v[n1] = buf[lane * 33 + n1];
    dft32<DIR>(v);
}

// Host side: emit(index, exponent) for the table of fft_warp1024, entry
// k1 * 32 + n1 = W1024^(n1 k1).
template <typename F>
inline void warp_twiddle_exponents(F&& emit) {
    for (int k1 = 0; k1 < 32; ++k1)
        for (int n1 = 0; n1 < 32; ++n1) emit(k1 * 32 + n1, n1 * k1);
}

}  // namespace ssg
