// ssg_noalloc.cu -- ssg_tendency_noalloc: the surface tendency for callers
// that cannot allocate device memory.
//
// Some callers cannot call cudaMalloc: code whose device memory is owned by
// someone else (a framework's caching allocator or memory pool that must
// account for every byte), and code inside a time-critical loop, where
// cudaMalloc may synchronize the device and stall for milliseconds.  For them
// this entry point computes compute_tendency! on device buffers they already
// own, and keeps its working storage in one file-scope device array that is
// part of the loaded library image.  It allocates nothing: no cudaMalloc, no
// cudaFree, no allocating library routine.
//
// The array holds the twiddle and wavenumber tables and the intermediate
// spectra of one call: SSG_NOALLOC_SCRATCH_BYTES (10 MiB), enough for grids up
// to 512 x 512.  Every GPU that loads the library holds these 10 MiB until the
// process exits.  Every call on a device uses the same array and leaves its
// contents behind; calls that overlap on that device (two streams, or two host
// threads) race on it and must be serialised by the caller.
//
// Each call writes the tables it uses into the array itself: a small kernel
// receives their values by value, as its launch parameters, and copies them
// in.  A call therefore depends on nothing an earlier call left behind.
#include "../../include/ssg_b200.h"
#include "kernels.cuh"
#include "fft.cuh"

#include <cmath>
#include <cstring>
#include <mutex>

using namespace ssg;

namespace {

constexpr size_t kScratchBytes = SSG_NOALLOC_SCRATCH_BYTES;
constexpr int kMaxDevices = 64;

// The working storage.  In host code this name is only a host-side handle:
// its device address comes from cudaGetSymbolAddress (per device, below).
static __device__ __align__(256) unsigned char g_tendency_scratch[kScratchBytes];

struct DeviceSlot {
    bool ready = false;
    unsigned char* base = nullptr;   // device address of g_tendency_scratch on this device
};

// The tables of one grid (N <= 512), passed by value to the kernel that
// writes them into the scratch array (12.3 KB of launch parameters).
constexpr int kMaxN = 512;
struct GridTables {
    int n, mx, my, pad;
    double2 tw[kMaxN];
    double kxc[2 * (kMaxN / 3)];
    double kyc[(2 * (kMaxN / 2 + 1)) / 3];
};

__global__ void __launch_bounds__(256) write_tables_kernel(const __grid_constant__ GridTables t, double2* tw,
                                                           double* kxc, double* kyc) {
    for (int i = threadIdx.x; i < t.n; i += blockDim.x) tw[i] = t.tw[i];
    for (int i = threadIdx.x; i < t.mx; i += blockDim.x) kxc[i] = t.kxc[i];
    for (int i = threadIdx.x; i < t.my; i += blockDim.x) kyc[i] = t.kyc[i];
}

std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];
// host-side cache of the last grid's table values (copied into each launch)
GridTables g_last_tables{};
double g_last_lx = 0.0, g_last_ly = 0.0;

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
    size_t tw, kxc, kyc, phih, bh, fh, P1, P2, P3, Q1, Q2, end;
};

Layout layout_for(const Dims& d) {
    Layout L{};
    size_t o = 0;
    L.tw = o;   o = align256(o + (size_t)d.N * sizeof(double2));
    L.kxc = o;  o = align256(o + (size_t)d.Mx * sizeof(double));
    L.kyc = o;  o = align256(o + (size_t)d.My * sizeof(double));
    L.phih = o; o = align256(o + d.c2() * sizeof(double2));
    L.bh = o;   o = align256(o + d.c2() * sizeof(double2));
    L.fh = o;   o = align256(o + d.c2() * sizeof(double2));
    L.P1 = o;   o = align256(o + d.m2() * sizeof(double2));
    L.P2 = o;   o = align256(o + d.m2() * sizeof(double2));
    L.P3 = o;   o = align256(o + d.m2() * sizeof(double2));
    L.Q1 = o;   o = align256(o + d.m2() * sizeof(double2));
    L.Q2 = o;   o = align256(o + d.m2() * sizeof(double2));
    L.end = o;
    return L;
}

// twiddles and compact wavenumbers, as ssg_ctx.cu builds them
void build_tables(const Dims& d, double lx, double ly, GridTables& t) {
    t.n = d.N;
    t.mx = d.Mx;
    t.my = d.My;
    double2* tw = t.tw;
    double* kxc = t.kxc;
    double* kyc = t.kyc;
    const long double PI_L = 3.141592653589793238462643383279502884L;
    for (int e = 0; e < d.N; ++e) tw[e] = make_double2(1.0, 0.0);
    pass_twiddle_exponents(d.N, [&](int i, int e) {
        const long double a = -2.0L * PI_L * (long double)e / (long double)d.N;
        tw[i] = make_double2((double)cosl(a), (double)sinl(a));
    });
    const double dx = lx / d.N, dy = ly / d.N;
    const double mulx = (1.0 / dx) / d.N, muly = (1.0 / dy) / d.N;
    const int nnx = (d.N - 1) / 2 + 1;
    for (int c = 0; c < d.Mx; ++c) {
        const int i = c < d.Kp ? c : c + (d.N - 2 * d.Kp);
        kxc[c] = 2.0 * M_PI * ((double)(i < nnx ? i : i - d.N) * mulx);
    }
    for (int j = 0; j < d.My; ++j) kyc[j] = 2.0 * M_PI * ((double)j * muly);
}

}  // namespace

// Declared in include/ssg_b200.h.  Compute the dealiased tendency
// -P J(phi_s, b_s) of compute_tendency! for device fields (nx*ny doubles,
// x fastest) on `stream`; asynchronous.  The first call on a device looks up
// the device address of the scratch array (cudaGetSymbolAddress); make that
// first call before any stream capture on that device.  Inputs are not
// checked for NaN or Inf: non-finite values propagate to dbdt.
extern "C" int ssg_tendency_noalloc(int32_t nx, int32_t ny, double lx, double ly, const double* phi_s,
                                    const double* b_s, double* dbdt, void* stream) {
    if (nx != ny || nx < 32 || nx > 512 || (nx & (nx - 1))) {
        set_global_error("ssg_tendency_noalloc: grid must be square, a power of two, 32 to 512 "
                         "(the static scratch array holds at most 512 x 512)");
        return SSG_ERR_ARG;
    }
    if (!(lx > 0 && ly > 0) || !phi_s || !b_s || !dbdt) {
        set_global_error("ssg_tendency_noalloc: null field pointer or non-positive domain length");
        return SSG_ERR_ARG;
    }
    Dims d{};
    d.N = nx;
    d.nyc = nx / 2 + 1;
    d.Kp = nx / 3;
    d.Mx = 2 * d.Kp;
    d.My = (2 * d.nyc) / 3;
    d.nz = 1;
    const Layout L = layout_for(d);
    if (L.end > kScratchBytes) {
        set_global_error("ssg_tendency_noalloc: grid does not fit the static scratch array");
        return SSG_ERR_ARG;
    }
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
        set_global_error("ssg_tendency_noalloc: no current CUDA device");
        return SSG_ERR_CUDA;
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    unsigned char* base = nullptr;
    static thread_local GridTables tables;
    {
        std::lock_guard<std::mutex> lock(g_mu);
        DeviceSlot& slot = g_slots[dev];
        if (!slot.ready) {
            void* p = nullptr;
            if (cudaGetSymbolAddress(&p, g_tendency_scratch) != cudaSuccess || !p) {
                set_global_error("ssg_tendency_noalloc: cudaGetSymbolAddress of the scratch array failed");
                return SSG_ERR_CUDA;
            }
            slot.base = static_cast<unsigned char*>(p);
            slot.ready = true;
        }
        base = slot.base;
        if (g_last_tables.n != nx || g_last_lx != lx || g_last_ly != ly) {
            build_tables(d, lx, ly, g_last_tables);
            g_last_lx = lx;
            g_last_ly = ly;
        }
        tables = g_last_tables;
    }
    auto at = [&](size_t off) { return base + off; };
    // this call's tables, written by a kernel that carries them as parameters
    write_tables_kernel<<<1, 256, 0, s>>>(tables, reinterpret_cast<double2*>(at(L.tw)),
                                          reinterpret_cast<double*>(at(L.kxc)), reinterpret_cast<double*>(at(L.kyc)));
    if (cudaGetLastError() != cudaSuccess) return SSG_ERR_CUDA;
    Tables tb{reinterpret_cast<const double2*>(at(L.tw)), nullptr, reinterpret_cast<const double*>(at(L.kxc)),
              reinterpret_cast<const double*>(at(L.kyc)), nullptr};
    double2* phih = reinterpret_cast<double2*>(at(L.phih));
    double2* bh = reinterpret_cast<double2*>(at(L.bh));
    double2* fh = reinterpret_cast<double2*>(at(L.fh));
    double2* P1 = reinterpret_cast<double2*>(at(L.P1));
    double2* P2 = reinterpret_cast<double2*>(at(L.P2));
    double2* P3 = reinterpret_cast<double2*>(at(L.P3));
    double2* Q1 = reinterpret_cast<double2*>(at(L.Q1));
    double2* Q2 = reinterpret_cast<double2*>(at(L.Q2));
    // physical fields -> compact spectra (the real fields' own spectra on the kept modes)
    if (launch_y_r2c(d, tb, phi_s, Q1, 1, s)) return SSG_ERR_CUDA;
    if (launch_x_fwd_compact(d, tb, Q1, phih, 1, 1.0, 0, s)) return SSG_ERR_CUDA;
    if (launch_y_r2c(d, tb, b_s, Q2, 1, s)) return SSG_ERR_CUDA;
    if (launch_x_fwd_compact(d, tb, Q2, bh, 1, 1.0, 0, s)) return SSG_ERR_CUDA;
    // the tendency, as in the time step
    if (launch_surf_xinv3(d, tb, phih, bh, P1, P2, P3, s)) return SSG_ERR_CUDA;
    if (launch_surf_y(d, tb, P1, P2, P3, Q1, Q2, s)) return SSG_ERR_CUDA;
    StageArgs a{};
    a.mode = STAGE_TENDENCY;   // writes fout only; no non-finite flag in this mode
    a.fout = fh;
    a.nonfinite = nullptr;
    if (launch_surf_xfwd_stage(d, tb, Q1, Q2, a, s)) return SSG_ERR_CUDA;
    // back to a physical field in the caller's buffer
    if (launch_x_inv_compact(d, tb, fh, P1, 1, 0, s)) return SSG_ERR_CUDA;
    if (launch_y_c2r(d, tb, P1, dbdt, 1, s)) return SSG_ERR_CUDA;
    return SSG_OK;
}
