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
#include "../../include/ssg_b200.h"
#include "kernels.cuh"
#include "fft.cuh"

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

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
    int n = 0;                       // grid whose tables are resident
    double lx = 0.0, ly = 0.0;
    std::vector<unsigned char> host_tables;  // kept alive for the table upload
};

std::mutex g_mu;
DeviceSlot g_slots[kMaxDevices];

size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }

struct Layout {
    size_t tw, kxc, kyc, flag, phih, bh, fh, P1, P2, P3, Q1, Q2, end;
};

Layout layout_for(const Dims& d) {
    Layout L{};
    size_t o = 0;
    L.tw = o;   o = align256(o + (size_t)d.N * sizeof(double2));
    L.kxc = o;  o = align256(o + (size_t)d.Mx * sizeof(double));
    L.kyc = o;  o = align256(o + (size_t)d.My * sizeof(double));
    L.flag = o; o = align256(o + sizeof(unsigned int));
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
void build_tables(const Dims& d, double lx, double ly, const Layout& L, std::vector<unsigned char>& out) {
    out.assign(L.flag, 0);
    double2* tw = reinterpret_cast<double2*>(out.data() + L.tw);
    double* kxc = reinterpret_cast<double*>(out.data() + L.kxc);
    double* kyc = reinterpret_cast<double*>(out.data() + L.kyc);
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
// first call before any stream capture on that device.
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
        if (slot.n != nx || slot.lx != lx || slot.ly != ly) {
            build_tables(d, lx, ly, L, slot.host_tables);
            if (cudaMemcpyAsync(base, slot.host_tables.data(), slot.host_tables.size(), cudaMemcpyHostToDevice, s) !=
                cudaSuccess)
                return SSG_ERR_CUDA;
            // pageable source: the copy is staged before cudaMemcpyAsync returns
            slot.n = nx;
            slot.lx = lx;
            slot.ly = ly;
        }
    }
    auto at = [&](size_t off) { return base + off; };
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
    unsigned int* flag = reinterpret_cast<unsigned int*>(at(L.flag));
    // the non-finite flag is accumulated with atomicOr: it must start at zero
    if (cudaMemsetAsync(flag, 0, sizeof(unsigned int), s) != cudaSuccess) return SSG_ERR_CUDA;
    // physical fields -> compact spectra (the real fields' own spectra on the kept modes)
    if (launch_y_r2c(d, tb, phi_s, Q1, 1, s)) return SSG_ERR_CUDA;
    if (launch_x_fwd_compact(d, tb, Q1, phih, 1, 1.0, 0, s)) return SSG_ERR_CUDA;
    if (launch_y_r2c(d, tb, b_s, Q2, 1, s)) return SSG_ERR_CUDA;
    if (launch_x_fwd_compact(d, tb, Q2, bh, 1, 1.0, 0, s)) return SSG_ERR_CUDA;
    // the tendency, as in the time step
    if (launch_surf_xinv3(d, tb, phih, bh, P1, P2, P3, s)) return SSG_ERR_CUDA;
    if (launch_surf_y(d, tb, P1, P2, P3, Q1, Q2, s)) return SSG_ERR_CUDA;
    StageArgs a{};
    a.mode = STAGE_TENDENCY;
    a.fout = fh;
    a.nonfinite = flag;
    if (launch_surf_xfwd_stage(d, tb, Q1, Q2, a, s)) return SSG_ERR_CUDA;
    // back to a physical field in the caller's buffer
    if (launch_x_inv_compact(d, tb, fh, P1, 1, 0, s)) return SSG_ERR_CUDA;
    if (launch_y_c2r(d, tb, P1, dbdt, 1, s)) return SSG_ERR_CUDA;
    return SSG_OK;
}
