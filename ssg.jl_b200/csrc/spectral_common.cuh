// spectral_common.cuh -- device helpers shared by the spectral kernel files:
// compact-mode indexing, packed real-pair transforms along y, the
// deterministic block reduction, cp.async wrappers, and the host-side launch
// helpers (launch counting, dynamic shared memory, dispatch on N).
#pragma once
#include "kernels.cuh"
#include "fft.cuh"

namespace ssg {

// compact column of full x-index i, or -1 when the 2/3 mask removes it
template <int N>
__device__ __forceinline__ int compact_col(int i) {
    constexpr int Kp = N / 3;
    return i < Kp ? i : (i >= N - Kp ? i - (N - 2 * Kp) : -1);
}

// Source of full x-index i in a compact row when the row holds a REAL field's
// spectrum.  The 2/3 mask keeps kx = -N/3 but not +N/3; in the ky = 0 row the
// two are conjugate partners, so (+N/3, 0) is read as conj of (-N/3, 0)
// (compact column N/3).  Returns -1 for masked-out modes.
template <int N>
__device__ __forceinline__ int real_src_col(int i, int ky, bool& conj_src) {
    int c = compact_col<N>(i);
    conj_src = false;
    if (c < 0 && ky == 0 && i == N / 3) {
        c = N / 3;
        conj_src = true;
    }
    return c;
}

// rows per block for x-passes: at least 128 threads per block
template <int N>
struct XRows {
    static constexpr int T = N / 8;
    static constexpr int R = (128 / T) > 1 ? (128 / T) : 1;
};

// column pairs per block for y-passes
template <int N, int THREADS>
struct YPairs {
    static constexpr int T = N / 8;
    static constexpr int P0 = THREADS / T > 0 ? THREADS / T : 1;
    static constexpr int P = P0 < N / 2 ? P0 : N / 2;
};

// Load the packed spectrum of two adjacent columns (x0, x0+1) of a mixed
// field with multiplier MULT applied, Hermitian-extended to the full ky
// range.  MULT: 0 -> 1, 1 -> -ky^2, 2 -> i ky, 3 -> -i ky.  The imaginary parts
// of the ky = 0 and ky = N/2 bins are dropped, as the complex-to-real
// transform does (rows up to My; My = N/2 + 1 for a full spectrum).
template <int N, int MULT, typename C>
__device__ __forceinline__ void load_c2r_pair(C (&v)[8], const C* __restrict__ X, int x0, int t, int My,
                                              const double* __restrict__ kyc) {
    using R = typename CT<C>::R;
    constexpr int T = N / 8;
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int k = t + p * T;
        int kk = -1;
        bool ext = false;
        if (k < My) {
            kk = k;
        } else if (k > N / 2 && N - k < My) {
            kk = N - k;
            ext = true;
        }
        C a = CT<C>::make(0, 0), b = CT<C>::make(0, 0);
        if (kk >= 0) {
            const C* row = X + (size_t)N * kk + x0;
            a = row[0];
            b = row[1];
            if constexpr (MULT == 1) {
                const R ky = (R)__ldg(&kyc[kk]);
                const R m = -(ky * ky);
                a = cscale(a, m);
                b = cscale(b, m);
            } else if constexpr (MULT == 2) {
                const R ky = (R)__ldg(&kyc[kk]);
                a = cmul_is(a, ky);
                b = cmul_is(b, ky);
            } else if constexpr (MULT == 3) {
                const R ky = -(R)__ldg(&kyc[kk]);
                a = cmul_is(a, ky);
                b = cmul_is(b, ky);
            }
            if (ext) {
                a = cconj(a);
                b = cconj(b);
            }
            if (k == 0 || k == N / 2) {  // the DC and Nyquist bins are real in a c2r
                a.y = 0;
                b.y = 0;
            }
        }
        v[p] = CT<C>::make(a.x - b.y, a.y + b.x);
    }
}

// Split the transform Z of z = d0 + i d1 into the half spectra of d0 and d1
// and store rows ky < My of the two columns.
template <int N, typename C>
__device__ __forceinline__ void store_r2c_pair(const C (&v)[8], C* buf, C* __restrict__ Y, int x0, int t, int My) {
    using R = typename CT<C>::R;
    constexpr int T = N / 8;
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 8; ++p) buf[fpad<C>(t + p * T)] = v[p];
    __syncthreads();
#pragma unroll
    for (int p = 0; p < 8; ++p) {
        const int k = t + p * T;
        if (k < My) {
            const C z = buf[fpad<C>(k)];
            const C zm = buf[fpad<C>((N - k) & (N - 1))];
            const R h = (R)0.5;
            const C a = CT<C>::make(h * (z.x + zm.x), h * (z.y - zm.y));
            const C b = CT<C>::make(h * (z.y + zm.y), -h * (z.x - zm.x));
            C* row = Y + (size_t)N * k + x0;
            row[0] = a;
            row[1] = b;
        }
    }
}

// Deterministic sum of two doubles over the block, then over blocks by the
// last block to finish (fixed order at both levels).
template <int TB>
__device__ __forceinline__ void block_reduce_pair(double ds, double ns, double* partials, unsigned int* ticket,
                                                  double* norms) {
    __shared__ double red[2][TB / 32];
    __shared__ bool is_last;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        ds += __shfl_down_sync(0xffffffffu, ds, off);
        ns += __shfl_down_sync(0xffffffffu, ns, off);
    }
    if (lane == 0) {
        red[0][warp] = ds;
        red[1][warp] = ns;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < TB / 32; ++w) {
            a += red[0][w];
            b += red[1][w];
        }
        partials[2 * blockIdx.x] = a;
        partials[2 * blockIdx.x + 1] = b;
        __threadfence();
        is_last = (atomicAdd(ticket, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!is_last) return;
    __threadfence();
    double a = 0.0, b = 0.0;
    for (int i = threadIdx.x; i < (int)gridDim.x; i += TB) {
        a += __ldcg(&partials[2 * i]);
        b += __ldcg(&partials[2 * i + 1]);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        a += __shfl_down_sync(0xffffffffu, a, off);
        b += __shfl_down_sync(0xffffffffu, b, off);
    }
    __syncthreads();
    if (lane == 0) {
        red[0][warp] = a;
        red[1][warp] = b;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double sa = 0.0, sb = 0.0;
        for (int w = 0; w < TB / 32; ++w) {
            sa += red[0][w];
            sb += red[1][w];
        }
        norms[0] = sa;
        norms[1] = sb;
        *ticket = 0u;
    }
}

// 16-byte asynchronous global -> shared copy (sm_80+ cp.async, L2 only)
__device__ __forceinline__ void cp_async16(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
// 8-byte asynchronous global -> shared copy (through L1)
__device__ __forceinline__ void cp_async8(void* smem_dst, const void* gmem_src) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem_dst);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem_src) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N_PENDING>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N_PENDING) : "memory"); }

// counts one launch (launch_counter) and reports a launch error
int record_launch();
static inline int check_launch() { return record_launch(); }

template <typename K>
static inline void set_smem(K kernel, size_t bytes) {
    if (bytes > 48 * 1024) cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N>
constexpr int tile_rows(int threads) {
    return threads / (N / 8) > 0 ? threads / (N / 8) : 1;
}
template <int N>
constexpr int tile_pairs(int threads) {
    return threads / (N / 8) < 1 ? 1 : (threads / (N / 8) > N / 2 ? N / 2 : threads / (N / 8));
}

// Call CALL with constexpr RR = rows (or pairs) per block for the block
// shape bt, one of the three candidates B0..B2; bt == 0 (or any other value),
// or N outside the tunable range, takes DEF.
#define SSG_DISPATCH_TILE(N_, bt, FN, DEF, B0, B1, B2, CALL)                                  \
    if constexpr ((N_) >= 64 && (N_) <= 512) {                                                \
        switch (bt) {                                                                         \
            case B0: { constexpr int RR = FN<N_>(B0); CALL; } break;                          \
            case B1: { constexpr int RR = FN<N_>(B1); CALL; } break;                          \
            case B2: { constexpr int RR = FN<N_>(B2); CALL; } break;                          \
            default: break;                                                                   \
        }                                                                                     \
    }                                                                                         \
    {                                                                                         \
        constexpr int RR = (DEF);                                                             \
        CALL;                                                                                 \
    }
#define SSG_DISPATCH_TILE_X(N_, bt, DEF, CALL) SSG_DISPATCH_TILE(N_, bt, tile_rows, DEF, 64, 128, 256, CALL)
#define SSG_DISPATCH_TILE_Y(N_, bt, DEF, CALL) SSG_DISPATCH_TILE(N_, bt, tile_pairs, DEF, 128, 256, 512, CALL)

#define SSG_DISPATCH_N(N_, CALL)                                            \
    switch (N_) {                                                           \
        case 8: { constexpr int NN = 8; CALL; } break;                      \
        case 16: { constexpr int NN = 16; CALL; } break;                    \
        case 32: { constexpr int NN = 32; CALL; } break;                    \
        case 64: { constexpr int NN = 64; CALL; } break;                    \
        case 128: { constexpr int NN = 128; CALL; } break;                  \
        case 256: { constexpr int NN = 256; CALL; } break;                  \
        case 512: { constexpr int NN = 512; CALL; } break;                  \
        case 1024: { constexpr int NN = 1024; CALL; } break;                \
        default: return -6;                                                 \
    }

}  // namespace ssg
